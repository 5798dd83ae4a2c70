// Discrete adjoint of the elastic RK stage (FP64, one block): the transpose
// of the curvilinear stage operator (derivative terms of every point in the
// conservative form of src/JU_xJU_yJU_z6.f90:12-809, face SATs of
// src/RHS_Interior.f90:1584-1768 with src/BoundaryConditions.f90:783-924,
// moment-tensor sources of src/moment_tensor.f90:875-1125) and of the
// Kennedy-Carpenter (5,4) low-storage update of src/time_step.f90:68-150.
// No counterpart in the reference, which has no adjoint.
//
// The right-hand side is L(F) = sum_a P_a D_a Q_a F + SAT(F): pointwise maps
// around one-dimensional SBP derivatives D_a along each axis.  Its transpose
// sum_a Q_a^T D_a^T P_a^T + SAT^T is evaluated as
//   * a pointwise pre-pass that turns the rate adjoint R into
//       Z_f = R_{v_f} / (rho J)                       (3 values)
//       Y_{a,f} = sum_r X_{r,a} W_{r,f}                (9 values)
//     with W = dsigma_dot / d(grad v) applied to R_sigma, and accumulates the
//     material gradient from the forward derivative terms of the stage input;
//   * a gather pass with the transposed derivative rows (tables built on the
//     host from the same coefficients as the forward rows):
//       Fbar_{v_f} += sum_a (1/h_a) D_a^T Y_{a,f}
//       Fbar_{sigma_{fr}} += J sum_a X_{r,a} (1/h_a) D_a^T Z_f
//   * a face pass: the SAT term is linear in the face point's fields (its
//     9 x 9 Jacobian, transposed) and its material derivatives come from
//     forward-mode dual numbers.
#pragma once

#include "wql3d_device.cuh"

namespace wql3d {

// adjoint buffers of one block (FP64, field layout of Blk)
struct AdjBlk {
  double *Fb, *DFb, *R;   // field / rate adjoints, rate adjoint of the current stage (9 comps each)
  double *ZY;             // pre-pass output: Z (3), Y (9)
  double *g;              // material gradient: lambda, mu, rho (3 comps)
  double *gM;             // moment-tensor gradient, nsrc x 6 (mxx myy mzz mxy mxz myz)
  double *S[5];           // stage inputs F^(0..4) of the step being reversed (9 comps each)
  const double *E[5];     // their derivative terms recorded by k_curv_fused (StageArgs::rec), or null
  const int *toff[3];     // transposed derivative rows per axis: [n][ADJ_TW] offsets
  const double *tc[3];    // ... and coefficients (0 pads)
  const double *res;      // receiver residuals of one sample, nrec x 3
};

constexpr int ADJ_TW = 12;  // taps of a transposed derivative row (<= 9 for traditional-6)

// forward-mode dual number a + eps b (eps^2 = 0): exact material derivatives
// of the SAT term
struct Dual {
  double a, b;
  __device__ Dual() : a(0), b(0) {}
  __device__ Dual(double x) : a(x), b(0) {}
  __device__ Dual(double x, double y) : a(x), b(y) {}
};
__device__ __forceinline__ Dual operator+(Dual x, Dual y) { return Dual(x.a + y.a, x.b + y.b); }
__device__ __forceinline__ Dual operator-(Dual x, Dual y) { return Dual(x.a - y.a, x.b - y.b); }
__device__ __forceinline__ Dual operator-(Dual x) { return Dual(-x.a, -x.b); }
__device__ __forceinline__ Dual operator*(Dual x, Dual y) { return Dual(x.a * y.a, x.a * y.b + x.b * y.a); }
__device__ __forceinline__ Dual operator/(Dual x, Dual y) {
  return Dual(x.a / y.a, (x.b * y.a - x.a * y.b) / (y.a * y.a));
}
__device__ __forceinline__ Dual any_sqrt(Dual x) {
  const double s = ::sqrt(x.a);
  return Dual(s, x.b / (2.0 * s));
}
__device__ __forceinline__ double any_sqrt(double x) { return ::sqrt(x); }

// SAT term pen * structure(bc_vector(u)) of one face point
// (src/RHS_Interior.f90:1584-1768, :2267-2287), generic in the number type
template <typename T>
__device__ void sat_term(int plus, const T u[9], T rho, T mu, T lam, const T l[3], const T m[3], const T n[3], T norm,
                         T r, T pen, T out[9]) {
  const T c_p = any_sqrt(((T)2.0 * mu + lam) / rho), c_s = any_sqrt(mu / rho);
  const T Zp = rho * c_p, Zs = rho * c_s;
  T ubc[9];
  bc_vector<T>(plus, u, Zs, Zp, r, l, m, n, norm, ubc);
  const T irho = (T)1.0 / rho;
  out[0] = pen * (irho * ubc[0]);
  out[1] = pen * (irho * ubc[1]);
  out[2] = pen * (irho * ubc[2]);
  out[3] = pen * (((T)2.0 * mu + lam) * ubc[3] + lam * (ubc[4] + ubc[5]));
  out[4] = pen * (((T)2.0 * mu + lam) * ubc[4] + lam * (ubc[3] + ubc[5]));
  out[5] = pen * (((T)2.0 * mu + lam) * ubc[5] + lam * (ubc[3] + ubc[4]));
  out[6] = pen * (mu * ubc[6]);
  out[7] = pen * (mu * ubc[7]);
  out[8] = pen * (mu * ubc[8]);
}

// host launchers (wql3d_adjoint.cu)
void adj_launch_stage(const Blk<double> &b, const AdjBlk &A, int stage, double Bdt, double A_s, cudaStream_t s,
                      int64_t *launches);
void adj_launch_moment(const Blk<double> &b, const AdjBlk &A, double t, cudaStream_t s, int64_t *launches);
void adj_launch_receivers(const Blk<double> &b, const AdjBlk &A, cudaStream_t s, int64_t *launches);
int upload_tables_adjoint(const void *t);

}  // namespace wql3d
