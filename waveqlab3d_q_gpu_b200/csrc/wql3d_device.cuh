// Device-side data model and kernels of the WaveQLab3D per-step volume update.
//
// Layout (HBM): every 3-D component is a padded x-fastest array with XOFF
// leading pad points in x (so the first interior point of every row starts on
// a 32-byte sector), a row pitch rounded up to 128 bytes, and 3 ghost planes
// in y and z.  Components of one logical array follow one another at a fixed
// component stride.  Two field buffers alternate between RK stages (the
// stencil reads buffer `cur` and the fused update writes buffer `cur^1`), so
// one stage is a single pass over F, DF and the material.
#pragma once

#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace wql3d {

constexpr int NB = 3;               // ghost width of the traditional-6 operator
constexpr int MESH_CART = 0;
constexpr int MESH_CURV = 1;
constexpr int RESP_EL = 0, RESP_Q4 = 1, RESP_Q8 = 2, RESP_FQ8 = 3;

// stage flags
constexpr int F_SCALE = 1;     // DF <- A*DF (and memory-variable / PML rates)
constexpr int F_RHS = 2;       // DF += L(F) (interior and near-boundary, anelastic, PML)
constexpr int F_SOURCE = 4;    // moment-tensor sources
constexpr int F_SAT = 8;       // physical-boundary SAT
constexpr int F_ISAT = 16;     // interface SAT (precomputed face vector)
constexpr int F_UPDATE = 32;   // F <- F + B*dt*DF (+ memory variables, PML)
constexpr int F_ALL = 63;

// Kennedy-Carpenter (5,4) coefficients, src/time_step.f90:53-62
__constant__ double c_rkA[5];
__constant__ double c_rkB[5];
__constant__ double c_rkC[6];

// SBP first-derivative rows 1..6 in the order the reference sums their terms
// (src/JU_xJU_yJU_z6.f90:74-161); [lit] selects the row-4 literal precision.
__constant__ int c_sbp_cnt[6];
__constant__ int c_sbp_idx[6][8];
__constant__ double c_sbp_c[2][6][8];

// 9-point discrete delta weights for alpha = 0, 25, 50, 100 (src/moment_tensor.f90:976-1121)
__constant__ double c_delta9[4][9] = {
    {-0.01171875, -0.03125, 0.046875, 0.28125, 0.4296875, 0.28125, 0.046875, -0.03125, -0.01171875},
    {-0.00246875, -0.02275, -0.014125, 0.16575, 0.4171875, 0.38675, 0.117875, -0.02975, -0.01846875},
    {-0.00728125, -0.028, 0.014875, 0.224, 0.4265625, 0.336, 0.081375, -0.032, -0.01553125},
    {-0.0095625, -0.02990625, 0.03053125, 0.25284375, 0.42890625, 0.30903125, 0.06384375, -0.03196875, -0.01371875}};

// F components staged in the interior kernel's shared plane
__constant__ int c_smf[8] = {0, 1, 2, 3, 4, 6, 7, 8};

struct DevSource {
  int type;
  int near[3];
  double phys[3];
  double par[11];  // duration t_init mxx myy mzz mxy mxz myz x y z
};

struct DevTime {
  double t;        // domain time at the start of the current step (D%t)
  int n;           // current step number (1-based)
  int nsamp;       // receiver samples taken
  int bad;         // first step whose station sample held a non-finite value (0: none)
  int stall;       // nonzero: a bounded wait in a stage kernel gave up (the stage's results are void)
};

template <typename T>
struct Blk {
  int nx, ny, nz;
  long long sy, sz;     // y and z strides in elements
  long long o1;         // element offset of point (1,1,1)
  long long vol;        // component stride
  T *F0, *F1;           // field buffers (9 components each)
  T *DF;                // rates (9 components)
  T *FC;                // FP32 path: Kahan compensation for F (9 components)
  T *G;                 // curvilinear: 18 derivative terms per point from k_curv_grad (see there)
  T *S6;                // curvilinear anelastic: per stress component the sum of the memory variables
  const double *X;      // physical coordinates x, y, z (FP64, field layout)
  int mms;              // manufactured-solution forcing and boundary data
  double mms_k[4];      // nt*pi, nx*pi, ny*pi, nz*pi
  T *M;                 // lambda, mu, rho
  // Cartesian: per-axis diagonal metric 1/X_a(i) (index 1..n)
  const T *mq, *mr, *ms;
  // curvilinear: metricx(1..3), metricy(1..3), metricz(1..3), then J
  const T *met;
  const T *J;
  int lo[3], hi[3];     // strict-interior bounds (1-based, inclusive)
  T hq, hr, hs;         // unit-cube spacing
  T ihq, ihr, ihs;      // 1/h
  T cx[3], cy[3], cz[3];// interior coefficients c/h
  int lit;              // SBP literal precision (index into c_sbp_c)
  int sep;              // Cartesian block whose metric is diagonal to roundoff (separable shell)
  const double *rowc;   // closure rows 0..11 (left 1..6, right n..n-5): 8 signed coefficients each
  const int *rowo;      // matching tap offsets relative to the point
  // derivative operator (WQL3D_FD_*): traditional-6, or an upwind pair
  // (forward D+ on the velocities, backward D- on the stresses) of closure
  // width uw.  Upwind rows, 16 slots each: D+ left 1..uw, D+ right n..n-uw+1,
  // D- left, D- right, then the near-boundary routine's D+ and D- interior
  // rows; urown holds each row's tap count, urowo the offsets from the point.
  int fd;
  int uw, utaps, uof, uob;   // width, interior taps, first interior offset of D+ / D-
  const double *urowc;
  const int *urowo;
  const int *urown;
  T ufw[3][10], ubw[3][10];  // strict-interior forward / backward coefficients over h per axis
  // open faces of an s-slab of a larger block (ghost planes hold the
  // neighbour's data): the central row applies up to the face on that axis
  int open_lo[3], open_hi[3];
  int nzg;              // s-planes of the whole block (nz unless a slab)
  // PML slabs (faces 0..5): box and Q / DQ (9 components each, slab-local)
  int npml;
  int pml_on[6];
  int pb[6][6];         // x0 x1 y0 y1 z0 z1
  long long pvol[6];
  T *Q[6], *DQ[6];
  T d0;                 // PML damping strength
  // anelastic memory variables: 6 components x nmech, stride vol
  int nmech;
  T *eta, *deta;
  const T *qs, *qp;
  T tau[8], w[8], ss[8], ps[8];
  T itau[8];            // 1/tau (the lean curvilinear update multiplies instead of dividing)
  int coarse;
  // physical boundaries
  int bc[6];
  T tau0;
  const T *nrm[6];      // curvilinear face bases n_l(3) n_m(3) n_n(3), face-local
  // interface SAT vectors (q-min face: isat[0], q-max face: isat[1]), 9 x ny*nz
  T *isat[2];
  // curvilinear lean path: face-SAT terms per face (tau0/h * structure(ubc) for
  // the rates, tau0/h * ubc for the face's PML slab), face-local (see k_curv_face_sat)
  T *fsat[6], *fdq[6];
  int foff[7];          // face offsets of the concatenated face launch
  // sources
  int nsrc, src_order, src_alpha, src_half;
  const DevSource *src;
  int sbox[6];          // union box of all source supports (x0 x1 y0 y1 z0 z1)
  // receivers
  int nrec;
  const int *ridx;
  double *seis;
  int max_samples;
};

struct StageArgs {
  int cur;              // field buffer read by the stencil
  int flags;
  int stage;            // 1..5
  double A, Bdt, dt;
  const DevTime *time;
  int pf = 0;           // k_curv_fused: 1 = L2 prefetch of the memory variables on entry
  // k_curv_fused: when set, every point writes the derivative terms of the
  // stage input the adjoint's material gradient needs (9 components, field
  // layout): e = (U0, U4, U8, U3 + U1, U6 + U2, U7 + U5) and the stress-flux
  // sums (S0 + S3 + S6, S1 + S4 + S7, S2 + S5 + S8)
  void *rec = nullptr;
  // Cartesian interior, TMA fills: 1 = issue no copies (test of the bounded
  // plane waits: they run out and the domain status reports the stall)
  int nofill = 0;
};

template <typename T>
__device__ __forceinline__ long long pidx(const Blk<T> &b, int x, int y, int z) {
  return b.o1 + (long long)(x - 1) + b.sy * (long long)(y - 1) + b.sz * (long long)(z - 1);
}

template <typename T>
__device__ __forceinline__ T ld(const T *p) { return __ldg(p); }

// L2 prefetch hint: pulls a line the kernel reads late towards the SM
// without holding a register for it
__device__ __forceinline__ void prefetch_l2(const void *p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// ---------------------------------------------------------------------------
// Asynchronous global -> shared copies (sm_80+ cp.async, still the lightest
// path for element-granular halo gathers on sm_100a).  src_size 0 zero-fills.
// ---------------------------------------------------------------------------
template <int BYTES>
__device__ __forceinline__ void cp_async(void *smem_dst, const void *gsrc, bool valid) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  int sz = valid ? BYTES : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(s), "l"(gsrc), "n"(BYTES), "r"(sz) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// ---------------------------------------------------------------------------
// Tensor-memory-accelerator (TMA) tile loads, cp.async.bulk.tensor, completing
// on an mbarrier in shared memory.  Each copy lands in the issuing CTA's own
// shared memory only, and every tensor map covers this GPU's own field
// arrays.  Rules the callers keep: the innermost
// coordinate times the element size is a multiple of 16 bytes, the shared
// destination is 128-byte aligned, and every wait is bounded.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// makes the initialised barriers visible to the async (TMA) proxy
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// the calling thread's arrival, announcing `bytes` of transfers to come
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// wait for phase `parity` of a barrier, giving up after `limit` polls
// (each poll may suspend the thread for a while); false when it gave up
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity, int limit) {
  for (int k = 0; k < limit; ++k)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
// one box of a 4-D tensor map (coordinates innermost first) into shared memory
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *tm, int c0, int c1, int c2, int c3,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], "
      "[%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
      : "memory");
}

// central (interior) SBP row at 1-based i of n points on axis a: 7 <= i <= n-6,
// or up to an open face of a slab
template <typename T>
__device__ __forceinline__ bool central_row(const Blk<T> &b, int a, int i, int n) {
  return (i >= 7 || b.open_lo[a]) && (i <= n - 6 || b.open_hi[a]);
}

// ---------------------------------------------------------------------------
// SBP stencil row at 1-based index i of an axis with n points: taps as
// relative offsets and signed coefficients, in the reference's summation
// order.  Interior rows (7 <= i <= n-6) use the central operator
// -1/60, 3/20, -3/4, 3/4, -3/20, 1/60 (src/JU_xJU_yJU_z6.f90:52-68).
// ---------------------------------------------------------------------------
struct Row {
  int cnt;
  int off[8];
  double c[8];
};

__device__ __forceinline__ void sbp_row(int i, int n, int lit, Row &r, bool open_lo = false, bool open_hi = false) {
  if ((i >= 7 || open_lo) && (i <= n - 6 || open_hi)) {
    r.cnt = 6;
    r.off[0] = -3; r.off[1] = -2; r.off[2] = -1; r.off[3] = 1; r.off[4] = 2; r.off[5] = 3;
    r.c[0] = -1.0 / 60.0; r.c[1] = 0.15; r.c[2] = -0.75; r.c[3] = 0.75; r.c[4] = -0.15; r.c[5] = 1.0 / 60.0;
    return;
  }
  if (i >= n - 5) {  // right closure: negated mirror of left row n+1-i
    int row = n - i;
    r.cnt = c_sbp_cnt[row];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      r.off[k] = (n + 1 - c_sbp_idx[row][k]) - i;
      r.c[k] = -c_sbp_c[lit][row][k];
    }
    return;
  }
  int row = i - 1;
  r.cnt = c_sbp_cnt[row];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    r.off[k] = c_sbp_idx[row][k] - i;
    r.c[k] = c_sbp_c[lit][row][k];
  }
}

// ---------------------------------------------------------------------------
// Moment-tensor source: src/moment_tensor.f90:813-1125
// ---------------------------------------------------------------------------
__device__ inline double source_time(int type, double t, double t0, double w) {
  const double pi = 3.141592653589793;
  switch (type) {
    case 0: return (w / (sqrt(2.0 * pi))) * exp((-(w * w) * ((t - t0) * (t - t0))) / 2.0);
    case 1: return (t / (w * w)) * exp(-t / w);
    case 2: return (w * w) * t * exp(-w * t);
    case 3: return (t < t0) ? (1.0 - cos(2.0 * pi * t / t0)) / t0 : 0.0;
    case 4: return ((t >= 0.0) && (t <= w)) ? 1.0 - cos(2.0 * pi * t / w) : 0.0;
    case 5: return (1.0 - (1.0 + t / w) * exp(-t / w));
    case 6: return (t <= w) ? t - w / (2.0 * pi) * sin(2.0 * pi * t / w) : w;
    case 7: {
      double a = pi * w * (t - t0);
      double a2 = a * a;
      return (1.0 - 2.0 * a2) * exp(-a2);
    }
  }
  return 0.0;
}

__device__ inline double singular_source(int i, int i0, double h, double a, int order, int alpha) {
  if (order == 2) {
    double beta = (1.0 - 2.0 * a) / 4.0 + 0.25;
    double gam = (2.0 * a - 1.0) / 16.0;
    double gap = (2.0 * a + 1.0) / 16.0;
    if (i == i0 - 2) return (-gam) / h;
    if (i == i0 - 1) return (beta + 3.0 * gam - gap) / h;
    if (i == i0) return (1.0 - a - 2.0 * beta - 3.0 * gam + 3.0 * gap) / h;
    if (i == i0 + 1) return (a + beta + gam - 3.0 * gap) / h;
    if (i == i0 + 2) return gap / h;
    return 0.0;
  }
  int k = i - i0;
  if (k < -4 || k > 4) return 0.0;
  int row = alpha == 0 ? 0 : alpha == 25 ? 1 : alpha == 50 ? 2 : alpha == 100 ? 3 : -1;
  if (row < 0) return 0.0;
  const double *w = c_delta9[row];
  return w[k + 4] / h;
}

// diagonal metric at a point (Cartesian: per-axis table; curvilinear: array)
template <typename T, int MESH>
__device__ __forceinline__ T diag_metric(const Blk<T> &b, int axis, int x, int y, int z, long long p) {
  return ld(b.met + (long long)(axis * 3 + axis) * b.vol + p);
}

template <typename T, int MESH>
__device__ void add_sources(const Blk<T> &b, double t, int x, int y, int z, long long p, T df[9]) {
  for (int i = 0; i < b.nsrc; ++i) {
    const DevSource &s = b.src[i];
    if (s.near[0] < 1) continue;
    if (abs(x - s.near[0]) > b.src_half || abs(y - s.near[1]) > b.src_half || abs(z - s.near[2]) > b.src_half) continue;
    double A = source_time(s.type, t, s.par[1], s.par[0]);
    double hx = (double)b.hq / (double)diag_metric<T, MESH>(b, 0, x, y, z, p);
    double hy = (double)b.hr / (double)diag_metric<T, MESH>(b, 1, x, y, z, p);
    double hz = (double)b.hs / (double)diag_metric<T, MESH>(b, 2, x, y, z, p);
    double ax = (s.par[8] - s.phys[0]) / hx;
    double ay = (s.par[9] - s.phys[1]) / hy;
    double az = (s.par[10] - s.phys[2]) / hz;
    double dx = singular_source(x, s.near[0], hx, ax, b.src_order, b.src_alpha);
    double dy = singular_source(y, s.near[1], hy, ay, b.src_order, b.src_alpha);
    double dz = singular_source(z, s.near[2], hz, az, b.src_order, b.src_alpha);
    double delta = dx * dy * dz;
#pragma unroll
    for (int c = 0; c < 6; ++c) df[3 + c] = (T)((double)df[3 + c] - A * s.par[2 + c] * delta);
  }
}

// ---------------------------------------------------------------------------
// Physical-boundary SAT at one face point: BC_* + BCm/BCp + structure,
// src/BoundaryConditions.f90:50-924, src/RHS_Interior.f90:1584-1768, :2267-2287
// ---------------------------------------------------------------------------
template <typename T>
__device__ void bc_vector(int plus, const T u[9], T Zs, T Zp, T r, const T l[3], const T m[3], const T n[3], T norm,
                          T ubc[9]) {
  T T0 = n[0] * u[3] + n[1] * u[6] + n[2] * u[7];
  T T1 = n[0] * u[6] + n[1] * u[4] + n[2] * u[8];
  T T2 = n[0] * u[7] + n[1] * u[8] + n[2] * u[5];
  T vl = l[0] * u[0] + l[1] * u[1] + l[2] * u[2];
  T vm = m[0] * u[0] + m[1] * u[1] + m[2] * u[2];
  T vn = n[0] * u[0] + n[1] * u[1] + n[2] * u[2];
  T Tl = l[0] * T0 + l[1] * T1 + l[2] * T2;
  T Tm = m[0] * T0 + m[1] * T1 + m[2] * T2;
  T Tn = n[0] * T0 + n[1] * T1 + n[2] * T2;
  const T one = (T)1, half = (T)0.5;
  T sg = plus ? one : -one;
  T pl = half * ((one - r) * Zs * vl + sg * ((one + r) * Tl));
  T pm = half * ((one - r) * Zs * vm + sg * ((one + r) * Tm));
  T pn = half * ((one - r) * Zp * vn + sg * ((one + r) * Tn));
  T ql = half * ((one - r) * vl + sg * ((one + r) / Zs * Tl));
  T qm = half * ((one - r) * vm + sg * ((one + r) / Zs * Tm));
  T qn = half * ((one - r) * vn + sg * ((one + r) / Zp * Tn));
  T Fx = l[0] * pl + m[0] * pm + n[0] * pn;
  T Fy = l[1] * pl + m[1] * pm + n[1] * pn;
  T Fz = l[2] * pl + m[2] * pm + n[2] * pn;
  T F_x = l[0] * ql + m[0] * qm + n[0] * qn;
  T F_y = l[1] * ql + m[1] * qm + n[1] * qn;
  T F_z = l[2] * ql + m[2] * qm + n[2] * qn;
  ubc[0] = norm * Fx;
  ubc[1] = norm * Fy;
  ubc[2] = norm * Fz;
  ubc[3] = sg * (norm * n[0] * F_x);
  ubc[4] = sg * (norm * n[1] * F_y);
  ubc[5] = sg * (norm * n[2] * F_z);
  ubc[6] = sg * (norm * (n[1] * F_x + n[0] * F_y));
  ubc[7] = sg * (norm * (n[2] * F_x + n[0] * F_z));
  ubc[8] = sg * (norm * (n[2] * F_y + n[1] * F_z));
}

// face bases of a diagonal-metric Cartesian block: gen_orth_vectors applied to
// the axis normals (src/unit_normals.f90:217-249)
template <typename T>
__device__ __forceinline__ void cart_basis(int axis, T l[3], T m[3], T n[3]) {
  for (int c = 0; c < 3; ++c) { l[c] = 0; m[c] = 0; n[c] = 0; }
  if (axis == 0) { n[0] = 1; m[1] = 1; l[2] = 1; }
  else if (axis == 1) { n[1] = 1; m[2] = 1; l[0] = 1; }
  else { n[2] = 1; m[1] = 1; l[0] = -1; }
}

// ---------------------------------------------------------------------------
// Manufactured solution (src/mms.f90:136-235): v = cos(nt pi t) sin sin sin,
// sigma = cos(nt pi t) cos cos cos
// ---------------------------------------------------------------------------
template <typename T>
__device__ void mms_exact(const Blk<T> &b, double t, long long p, double u[9]) {
  const double X0 = b.X[p], X1 = b.X[b.vol + p], X2 = b.X[2 * b.vol + p];
  const double ct = cos(b.mms_k[0] * t);
  const double a = sin(b.mms_k[1] * X0) * sin(b.mms_k[2] * X1) * sin(b.mms_k[3] * X2);
  const double c = cos(b.mms_k[1] * X0) * cos(b.mms_k[2] * X1) * cos(b.mms_k[3] * X2);
#pragma unroll
  for (int k = 0; k < 3; ++k) u[k] = ct * a;
#pragma unroll
  for (int k = 3; k < 9; ++k) u[k] = ct * c;
}

// rates -= L(u*) - u*_t (mms_forcing, src/mms.f90:77-134)
template <typename T>
__device__ void mms_forcing(const Blk<T> &b, double t, long long p, T df[9]) {
  const double X0 = b.X[p], X1 = b.X[b.vol + p], X2 = b.X[2 * b.vol + p];
  const double kt = b.mms_k[0], kx = b.mms_k[1], ky = b.mms_k[2], kz = b.mms_k[3];
  const double ct = cos(kt * t), st = sin(kt * t);
  const double sx = sin(kx * X0), cx = cos(kx * X0), sy = sin(ky * X1), cy = cos(ky * X1);
  const double sz = sin(kz * X2), cz = cos(kz * X2);
  // velocity components 0-2 share one profile, stresses 3-8 another
  const double vt = -kt * st * sx * sy * sz, vx = kx * ct * cx * sy * sz, vy = ky * ct * sx * cy * sz,
               vz = kz * ct * sx * sy * cz;
  const double st_ = -kt * st * cx * cy * cz, sx_ = -kx * ct * sx * cy * cz, sy_ = -ky * ct * cx * sy * cz,
               sz_ = -kz * ct * cx * cy * sz;
  const double lam = (double)b.M[p], mu = (double)b.M[b.vol + p], rho = (double)b.M[2 * b.vol + p];
  double f[9];
  f[0] = (1.0 / rho) * (sx_ + sy_ + sz_);
  f[1] = (1.0 / rho) * (sx_ + sy_ + sz_);
  f[2] = (1.0 / rho) * (sx_ + sy_ + sz_);
  f[3] = (2.0 * mu + lam) * vx + lam * vy + lam * vz;
  f[4] = lam * vx + (2.0 * mu + lam) * vy + lam * vz;
  f[5] = lam * vx + lam * vy + (2.0 * mu + lam) * vz;
  f[6] = mu * (vy + vx);
  f[7] = mu * (vz + vx);
  f[8] = mu * (vz + vy);
#pragma unroll
  for (int c = 0; c < 9; ++c) df[c] = df[c] - (T)(f[c] - (c < 3 ? vt : st_));
}

template <typename T, int MESH, bool SEP>
__device__ void add_face_sats(const Blk<T> &b, const T *F, int x, int y, int z, long long p, T df[9], bool pml_point,
                              double t) {
  const int pos[3] = {x, y, z};
  const int nn[3] = {b.nx, b.ny, b.nz};
  T u[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) u[c] = F[c * b.vol + p];
  if (b.mms) {
    // u - switch * fu with the exact solution (src/BoundaryConditions.f90:84-88)
    double fu[9];
    mms_exact<T>(b, t, p, fu);
#pragma unroll
    for (int c = 0; c < 9; ++c) u[c] = (T)((double)u[c] - fu[c]);
  }
  const T lam = b.M[p], mu = b.M[b.vol + p], rho = b.M[2 * b.vol + p];
  for (int f = 0; f < 6; ++f) {
    int type = b.bc[f];
    if (type <= 0) continue;
    int axis = f >> 1, plus = f & 1;
    if (pos[axis] != (plus ? nn[axis] : 1)) continue;
    T r = type == 1 ? (T)0 : type == 2 ? (T)1 : (T)-1;
    T c_p = sqrt(((T)2 * mu + lam) / rho);
    T c_s = sqrt(mu / rho);
    T Zp = rho * c_p, Zs = rho * c_s;
    T l[3], m[3], n[3], norm;
    if (SEP) {
      cart_basis(axis, l, m, n);
      norm = axis == 0 ? ld(b.mq + x) : axis == 1 ? ld(b.mr + y) : ld(b.ms + z);
    } else {
      T qx = ld(b.met + (long long)(0 + axis) * b.vol + p);
      T qy = ld(b.met + (long long)(3 + axis) * b.vol + p);
      T qz = ld(b.met + (long long)(6 + axis) * b.vol + p);
      norm = sqrt(qx * qx + qy * qy + qz * qz);
      int a0 = axis == 0 ? y : x, a1 = axis == 2 ? y : z;
      int d0 = axis == 0 ? b.ny : b.nx;
      long long fp = (long long)(a0 - 1) + (long long)d0 * (a1 - 1);
      long long fn = (long long)d0 * (axis == 2 ? b.ny : b.nz);
      const T *B = b.nrm[f];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        l[c] = ld(B + (0 + c) * fn + fp);
        m[c] = ld(B + (3 + c) * fn + fp);
        n[c] = ld(B + (6 + c) * fn + fp);
      }
    }
    T ubc[9], Ux[9];
    bc_vector<T>(plus, u, Zs, Zp, r, l, m, n, norm, ubc);
    // structure(), src/RHS_Interior.f90:2267-2287
    const T irho = (T)1 / rho;
    Ux[0] = irho * ubc[0];
    Ux[1] = irho * ubc[1];
    Ux[2] = irho * ubc[2];
    Ux[3] = ((T)2 * mu + lam) * ubc[3] + lam * (ubc[4] + ubc[5]);
    Ux[4] = ((T)2 * mu + lam) * ubc[4] + lam * (ubc[3] + ubc[5]);
    Ux[5] = ((T)2 * mu + lam) * ubc[5] + lam * (ubc[3] + ubc[4]);
    Ux[6] = mu * ubc[6];
    Ux[7] = mu * ubc[7];
    Ux[8] = mu * ubc[8];
    T h = axis == 0 ? b.hq : axis == 1 ? b.hr : b.hs;
    T pen = b.tau0 / h;
#pragma unroll
    for (int c = 0; c < 9; ++c) df[c] = df[c] - pen * Ux[c];
    if (pml_point && b.pml_on[f]) {
      const int *B = b.pb[f];
      long long q = (long long)(x - B[0]) + (long long)(B[1] - B[0] + 1) * ((long long)(y - B[2]) + (long long)(B[3] - B[2] + 1) * (long long)(z - B[4]));
      T *DQ = b.DQ[f];
#pragma unroll
      for (int c = 0; c < 9; ++c) DQ[c * b.pvol[f] + q] = DQ[c * b.pvol[f] + q] - pen * ubc[c];
    }
  }
}

// ---------------------------------------------------------------------------
// Anelastic memory variables at one point, src/RHS_Interior.f90:2599-2908,
// :3361-3477 and the interior copies src/JU_xJU_yJU_z6.f90:16263-16420.
// e = (exx, eyy, ezz, gxy, gxz, gyz) strain rates (PML-corrected in slabs).
// The eta sums are subtracted from s (df in the interior form, DU near
// boundaries).  Memory-variable rates are scaled, accumulated and (with
// F_UPDATE) integrated here because they are point-local.
// ---------------------------------------------------------------------------
template <typename T, int RESP>
__device__ void anelastic_point(const Blk<T> &b, const StageArgs &a, int x, int y, int z, long long p, const T e[6], T tr,
                                T s[9], bool do_rhs) {
  constexpr int N = RESP == RESP_Q4 ? 4 : 8;
  const long long V = b.vol;
  const T lam = b.M[p], mu = b.M[V + p];
  T qs = 0, qp = 0;
  if (RESP != RESP_FQ8) { qs = ld(b.qs + p); qp = ld(b.qp + p); }
  int active = 1 + ((x - 1) & 1) + 2 * ((y - 1) & 1) + 4 * ((z - 1) & 1);
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    T eta[N], de[N];
#pragma unroll
    for (int i = 0; i < N; ++i) {
      eta[i] = b.eta[(long long)(c * N + i) * V + p];
      de[i] = b.deta[(long long)(c * N + i) * V + p];
      if (a.flags & F_SCALE) de[i] = (T)a.A * de[i];
    }
    if (do_rhs) {
      T sum = eta[0];
#pragma unroll
      for (int i = 1; i < N; ++i) sum = sum + eta[i];
      s[3 + c] = s[3 + c] - sum;
#pragma unroll
      for (int i = 0; i < N; ++i) {
        if (RESP == RESP_FQ8) {
          if (b.coarse && (i + 1) != active) continue;
          T ss = b.ss[i], ps = b.ps[i];
          if (c < 3)
            de[i] = de[i] + (((ss * (T)2 * mu) * e[c] + ((lam + (T)2 * mu) * ps - (T)2 * mu * ss) * tr) - eta[i]) / b.tau[i];
          else
            de[i] = de[i] + ((ss * mu * e[c] - eta[i]) / b.tau[i]);
        } else {
          T w = b.w[i];
          if (c < 3)
            de[i] = de[i] + (((w * (T)2 * mu * qs) * e[c] + (w * ((lam + (T)2 * mu) * qp - (T)2 * mu * qs)) * tr) - eta[i]) / b.tau[i];
          else
            de[i] = de[i] + ((w * mu * qs * e[c] - eta[i]) / b.tau[i]);
        }
      }
    }
#pragma unroll
    for (int i = 0; i < N; ++i) {
      b.deta[(long long)(c * N + i) * V + p] = de[i];
      if (a.flags & F_UPDATE) b.eta[(long long)(c * N + i) * V + p] = eta[i] + (T)a.Bdt * de[i];
    }
  }
}

// ---------------------------------------------------------------------------
// PML at one point, src/RHS_Interior.f90:1846-2265.  Slabs are visited in the
// reference order z-, z+, y-, y+, x-, x+.  Ux(4:9) carry J (JJU_x6), so the
// DQ(1:3) sources divide by J.
// ---------------------------------------------------------------------------
template <typename T, bool JFORM>
__device__ void pml_point(const Blk<T> &b, const StageArgs &a, int x, int y, int z, long long p, const T Ux[9], const T Uy[9],
                          const T Uz[9], T rhoJ_inv, T lambda2mu, T J, T DU[9]) {
  const int order[6] = {4, 5, 2, 3, 0, 1};
  const long long V = b.vol;
  const T lam = b.M[p], mu = b.M[V + p];
  const T cfs = (T)1;
  const int pos[3] = {x, y, z};
  for (int oi = 0; oi < 6; ++oi) {
    int f = order[oi];
    if (!b.pml_on[f]) continue;
    const int *B = b.pb[f];
    if (x < B[0] || x > B[1] || y < B[2] || y > B[3] || z < B[4] || z > B[5]) continue;
    int axis = f >> 1;
    int n = axis == 0 ? b.nx : axis == 1 ? b.ny : b.nz;
    int i = pos[axis];
    T v = (f == 4) ? (T)(i - b.npml) : ((f & 1) ? (T)(i - (n - b.npml)) : (T)(i - (1 + b.npml)));
    T d = b.d0 * fabs(v / (T)b.npml);
    long long q = (long long)(x - B[0]) + (long long)(B[1] - B[0] + 1) * ((long long)(y - B[2]) + (long long)(B[3] - B[2] + 1) * (long long)(z - B[4]));
    T *Qp = b.Q[f];
    T *DQp = b.DQ[f];
    const long long PV = b.pvol[f];
    T Q[9], DQ[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) {
      Q[c] = Qp[c * PV + q];
      DQ[c] = DQp[c * PV + q];
    }
    if (JFORM) {
      DU[0] = DU[0] - d * J * Q[0] * rhoJ_inv;
      DU[1] = DU[1] - d * J * Q[1] * rhoJ_inv;
      DU[2] = DU[2] - d * J * Q[2] * rhoJ_inv;
    } else {
      DU[0] = DU[0] - d * Q[0] * rhoJ_inv;
      DU[1] = DU[1] - d * Q[1] * rhoJ_inv;
      DU[2] = DU[2] - d * Q[2] * rhoJ_inv;
    }
    DU[3] = DU[3] - d * (lambda2mu * Q[3] + lam * Q[4] + lam * Q[5]);
    DU[4] = DU[4] - d * (lam * Q[3] + lambda2mu * Q[4] + lam * Q[5]);
    DU[5] = DU[5] - d * (lam * Q[3] + lam * Q[4] + lambda2mu * Q[5]);
    DU[6] = DU[6] - mu * d * Q[6];
    DU[7] = DU[7] - mu * d * Q[7];
    DU[8] = DU[8] - mu * d * Q[8];
    T src[9];
    const T iJ = JFORM ? J : (T)1;
    if (axis == 2) {
      src[0] = Uz[7] / iJ; src[1] = Uz[8] / iJ; src[2] = Uz[5] / iJ; src[3] = 0; src[4] = 0;
      src[5] = Uz[2]; src[6] = 0; src[7] = Uz[0]; src[8] = Uz[1];
    } else if (axis == 1) {
      src[0] = Uy[6] / iJ; src[1] = Uy[4] / iJ; src[2] = Uy[8] / iJ; src[3] = 0; src[4] = Uy[1];
      src[5] = 0; src[6] = Uy[0]; src[7] = 0; src[8] = Uy[2];
    } else {
      src[0] = Ux[3] / iJ; src[1] = Ux[6] / iJ; src[2] = Ux[7] / iJ; src[3] = Ux[0]; src[4] = 0;
      src[5] = 0; src[6] = Ux[1]; src[7] = Ux[2]; src[8] = 0;
    }
#pragma unroll
    for (int c = 0; c < 9; ++c) DQ[c] = DQ[c] + src[c] - (d + cfs) * Q[c];
#pragma unroll
    for (int c = 0; c < 9; ++c) DQp[c * PV + q] = DQ[c];
  }
}

// PML damping and auxiliary fields for the anelastic strain correction,
// src/RHS_Interior.f90:2351-2451
template <typename T>
__device__ bool pml_strain_correction(const Blk<T> &b, int x, int y, int z, T e[6]) {
  bool in = false;
  T dd[3] = {0, 0, 0};
  T Qd[3][9];
  for (int k = 0; k < 3; ++k)
    for (int c = 0; c < 9; ++c) Qd[k][c] = 0;
  const int pos[3] = {x, y, z};
  for (int f = 0; f < 6; ++f) {
    if (!b.pml_on[f]) continue;
    const int *B = b.pb[f];
    if (x < B[0] || x > B[1] || y < B[2] || y > B[3] || z < B[4] || z > B[5]) continue;
    in = true;
    int axis = f >> 1;
    int n = axis == 0 ? b.nx : axis == 1 ? b.ny : b.nz;
    int i = pos[axis];
    T v = (f == 4) ? (T)(i - b.npml) : ((f & 1) ? (T)(i - (n - b.npml)) : (T)(i - (1 + b.npml)));
    dd[axis] = b.d0 * fabs(v / (T)b.npml);
    long long q = (long long)(x - B[0]) + (long long)(B[1] - B[0] + 1) * ((long long)(y - B[2]) + (long long)(B[3] - B[2] + 1) * (long long)(z - B[4]));
    for (int c = 0; c < 9; ++c) Qd[axis][c] = b.Q[f][c * b.pvol[f] + q];
  }
  if (!in) return false;
  // exx = Ux(1) - dx*Qx(4), ..., gxy = (Uy(1)+Ux(2)) - dx*Qx(7) - dy*Qy(7), ...
  e[0] = e[0] - dd[0] * Qd[0][3];
  e[1] = e[1] - dd[1] * Qd[1][4];
  e[2] = e[2] - dd[2] * Qd[2][5];
  e[3] = e[3] - dd[0] * Qd[0][6] - dd[1] * Qd[1][6];
  e[4] = e[4] - dd[0] * Qd[0][7] - dd[2] * Qd[2][7];
  e[5] = e[5] - dd[1] * Qd[1][8] - dd[2] * Qd[2][8];
  return true;
}

// ---------------------------------------------------------------------------
// Near-boundary derivatives, both mesh kinds: JJU_x6
// (src/JU_xJU_yJU_z6.f90:12-809) for one metric row: velocities
// X_a(p) * D_a(u), stresses D_a(F * J * X_a), summed over the three axes.
// A Cartesian grid keeps its full metric here: without -r8 the row-4
// literal leaves off-diagonal metric terms of order 1e-10.
// ---------------------------------------------------------------------------
template <typename T>
__device__ void jju6_row(const Blk<T> &b, const T *F, int x, int y, int z, long long p, int mrow, T Ju[9]) {
  const int pos[3] = {x, y, z};
  const int nn[3] = {b.nx, b.ny, b.nz};
  const long long st[3] = {1, b.sy, b.sz};
  const T ih[3] = {b.ihq, b.ihr, b.ihs};
  for (int f = 0; f < 9; ++f) Ju[f] = 0;
  for (int a = 0; a < 3; ++a) {
    Row r;
    sbp_row(pos[a], nn[a], b.lit, r, b.open_lo[a], b.open_hi[a]);
    const T *X = b.met + (long long)(mrow * 3 + a) * b.vol;
    T sv[3] = {0, 0, 0};
    T ss[6] = {0, 0, 0, 0, 0, 0};
    for (int k = 0; k < r.cnt; ++k) {
      long long q = p + (long long)r.off[k] * st[a];
      T c = (T)r.c[k];
      T JX = ld(b.J + q);
      T Xq = ld(X + q);
#pragma unroll
      for (int f = 0; f < 3; ++f) sv[f] = sv[f] + c * ld(F + f * b.vol + q);
#pragma unroll
      for (int f = 0; f < 6; ++f) ss[f] = ss[f] + c * ld(F + (3 + f) * b.vol + q) * JX * Xq;
    }
    T Xp = ld(X + p);
#pragma unroll
    for (int f = 0; f < 3; ++f) Ju[f] = Ju[f] + ih[a] * (Xp * sv[f]);
#pragma unroll
    for (int f = 0; f < 6; ++f) Ju[3 + f] = Ju[3 + f] + ih[a] * ss[f];
  }
}

// One tap of the near-boundary operator for all three metric rows:
// velocities accumulate sum c*F; stresses accumulate ((c*F)*J)*X_row,a per row
// (the reference's association, src/JU_xJU_yJU_z6.f90:52-68).
template <typename T>
__device__ __forceinline__ void jju_tap(const Blk<T> &b, const T *F, long long q, int a, T c, T sv[3], T acc[3][6]) {
  const long long V = b.vol;
  const T Jq = ld(b.J + q);
  const T X0 = ld(b.met + (long long)(0 * 3 + a) * V + q);
  const T X1 = ld(b.met + (long long)(1 * 3 + a) * V + q);
  const T X2 = ld(b.met + (long long)(2 * 3 + a) * V + q);
#pragma unroll
  for (int f = 0; f < 3; ++f) sv[f] = sv[f] + c * ld(F + f * V + q);
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    const T cFJ = c * ld(F + (3 + f) * V + q) * Jq;
    acc[0][f] = acc[0][f] + cFJ * X0;
    acc[1][f] = acc[1][f] + cFJ * X1;
    acc[2][f] = acc[2][f] + cFJ * X2;
  }
}

// Near-boundary derivatives of all nine fields for the three metric rows:
// U[row][f] = JJU_x6 with X = metricx / metricy / metricz (src/JU_xJU_yJU_z6.f90:12-809).
template <typename T>
__device__ void jju6_all(const Blk<T> &b, const T *F, int x, int y, int z, long long p, T U[3][9]) {
  const int pos[3] = {x, y, z};
  const int nn[3] = {b.nx, b.ny, b.nz};
  const long long st[3] = {1, b.sy, b.sz};
  const T ih[3] = {b.ihq, b.ihr, b.ihs};
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int f = 0; f < 9; ++f) U[r][f] = 0;
#pragma unroll 1
  for (int a = 0; a < 3; ++a) {
    T sv[3] = {0, 0, 0};
    T acc[3][6];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int f = 0; f < 6; ++f) acc[r][f] = 0;
    const int i = pos[a], n = nn[a];
    if (central_row(b, a, i, n)) {
      const T cc[6] = {(T)(-1.0 / 60.0), (T)0.15, (T)-0.75, (T)0.75, (T)-0.15, (T)(1.0 / 60.0)};
      const int off[6] = {-3, -2, -1, 1, 2, 3};
#pragma unroll
      for (int k = 0; k < 6; ++k) jju_tap(b, F, p + (long long)off[k] * st[a], a, cc[k], sv, acc);
    } else {
      const int row = i <= 6 ? i - 1 : 6 + (n - i);
      const double *rc = b.rowc + row * 8;
      const int *ro = b.rowo + row * 8;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const T c = (T)__ldg(rc + k);
        if (c != (T)0) jju_tap(b, F, p + (long long)__ldg(ro + k) * st[a], a, c, sv, acc);
      }
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const T Xp = ld(b.met + (long long)(r * 3 + a) * b.vol + p);
#pragma unroll
      for (int f = 0; f < 3; ++f) U[r][f] = U[r][f] + ih[a] * (Xp * sv[f]);
#pragma unroll
      for (int f = 0; f < 6; ++f) U[r][3 + f] = U[r][3 + f] + ih[a] * acc[r][f];
    }
  }
}

// Device row of the block's upwind operator D+ (plus) or D- at 1-based i of
// n points: closures from the left / right rows (the right rows win where
// both apply, n < 2w, as the reference assigns them last), the
// near-boundary routine's interior row elsewhere (the layout of Blk::urowc).
template <typename T>
__device__ __forceinline__ int up_row(const Blk<T> &b, bool plus, int i, int n) {
  const int w = b.uw;
  if (i > n - w) return (plus ? w : 3 * w) + (n - i);
  if (i <= w) return (plus ? 0 : 2 * w) + (i - 1);
  return 4 * w + (plus ? 0 : 1);
}

// Near-boundary upwind derivatives of all nine fields for the three metric
// rows (JJU_x4_upwind, JJU_x6_upwind, JJU_x6_upwind_drp of
// src/JU_xJU_yJU_z6.f90): velocities X_r,a(p) * D+_a(u), stresses
// D-_a(X_r,a J s) with each term associated as ((c X) J) s.
template <typename T>
__device__ void jju_up_all(const Blk<T> &b, const T *F, int x, int y, int z, long long p, T U[3][9]) {
  const int pos[3] = {x, y, z};
  const int nn[3] = {b.nx, b.ny, b.nz};
  const long long st[3] = {1, b.sy, b.sz};
  const T ih[3] = {b.ihq, b.ihr, b.ihs};
  const long long V = b.vol;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int f = 0; f < 9; ++f) U[r][f] = 0;
#pragma unroll 1
  for (int a = 0; a < 3; ++a) {
    const int rp = up_row(b, true, pos[a], nn[a]), rm = up_row(b, false, pos[a], nn[a]);
    T sv[3] = {0, 0, 0};
    const int np = __ldg(b.urown + rp);
    for (int k = 0; k < np; ++k) {
      const T c = (T)__ldg(b.urowc + rp * 16 + k);
      const long long q = p + (long long)__ldg(b.urowo + rp * 16 + k) * st[a];
#pragma unroll
      for (int f = 0; f < 3; ++f) sv[f] = sv[f] + c * ld(F + f * V + q);
    }
    T acc[3][6];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int f = 0; f < 6; ++f) acc[r][f] = 0;
    const int nm = __ldg(b.urown + rm);
    for (int k = 0; k < nm; ++k) {
      const T c = (T)__ldg(b.urowc + rm * 16 + k);
      const long long q = p + (long long)__ldg(b.urowo + rm * 16 + k) * st[a];
      const T Jq = ld(b.J + q);
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        const T cXJ = (c * ld(b.met + (long long)(r * 3 + a) * V + q)) * Jq;
#pragma unroll
        for (int f = 0; f < 6; ++f) acc[r][f] = acc[r][f] + cXJ * ld(F + (3 + f) * V + q);
      }
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const T Xp = ld(b.met + (long long)(r * 3 + a) * V + p);
#pragma unroll
      for (int f = 0; f < 3; ++f) U[r][f] = U[r][f] + ih[a] * (Xp * sv[f]);
#pragma unroll
      for (int f = 0; f < 6; ++f) U[r][3 + f] = U[r][3 + f] + ih[a] * acc[r][f];
    }
  }
}

// Strict-interior upwind derivative terms (JJU_x4_interior_upwind,
// src/JU_xJU_yJU_z6.f90:17865-18400; JJU_x6_interior_upwind, :18958-19510;
// JJU_x6_interior_upwind_drp): forward differences of the velocities at
// offsets uof .., backward of the stresses at uob ..; Cartesian with the
// diagonal metric at the point, curvilinear with the metric at the point for
// the velocities and (s X) J at the taps for the stresses.
template <typename T, int MESH>
__device__ __forceinline__ void up_interior(const Blk<T> &b, const T *F, int x, int y, int z, long long p, T DFx[9],
                                             T DFy[9], T DFz[9]) {
  const long long V = b.vol;
  const long long st[3] = {1, b.sy, b.sz};
  if (MESH == MESH_CART) {
    const T mx = ld(b.mq + x), my = ld(b.mr + y), mz = ld(b.ms + z);
#pragma unroll 1
    for (int k = 0; k < b.utaps; ++k) {
      const long long s = b.uof + k, t = b.uob + k;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const T *Fc = F + c * V;
        DFx[c] = DFx[c] + mx * b.ufw[0][k] * ld(Fc + p + s * st[0]);
        DFy[c] = DFy[c] + my * b.ufw[1][k] * ld(Fc + p + s * st[1]);
        DFz[c] = DFz[c] + mz * b.ufw[2][k] * ld(Fc + p + s * st[2]);
      }
#pragma unroll
      for (int c = 3; c < 9; ++c) {
        const T *Fc = F + c * V;
        DFx[c] = DFx[c] + mx * b.ubw[0][k] * ld(Fc + p + t * st[0]);
        DFy[c] = DFy[c] + my * b.ubw[1][k] * ld(Fc + p + t * st[1]);
        DFz[c] = DFz[c] + mz * b.ubw[2][k] * ld(Fc + p + t * st[2]);
      }
    }
  } else {
    T mp[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) mp[k] = ld(b.met + k * V + p);
#pragma unroll 1
    for (int k = 0; k < b.utaps; ++k) {
      const long long s = b.uof + k, t = b.uob + k;
      const long long q0 = p + s * st[0], q1 = p + s * st[1], q2 = p + s * st[2];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const T *Fc = F + c * V;
        const T f0 = ld(Fc + q0), f1 = ld(Fc + q1), f2 = ld(Fc + q2);
        DFx[c] = DFx[c] + mp[0] * b.ufw[0][k] * f0 + mp[1] * b.ufw[1][k] * f1 + mp[2] * b.ufw[2][k] * f2;
        DFy[c] = DFy[c] + mp[3] * b.ufw[0][k] * f0 + mp[4] * b.ufw[1][k] * f1 + mp[5] * b.ufw[2][k] * f2;
        DFz[c] = DFz[c] + mp[6] * b.ufw[0][k] * f0 + mp[7] * b.ufw[1][k] * f1 + mp[8] * b.ufw[2][k] * f2;
      }
      const long long r0 = p + t * st[0], r1 = p + t * st[1], r2 = p + t * st[2];
      const T J0 = ld(b.J + r0), J1 = ld(b.J + r1), J2 = ld(b.J + r2);
      T m0[3], m1[3], m2[3];  // metric row r, q- / r- / s-entry at the backward taps
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        m0[r] = ld(b.met + (r * 3 + 0) * V + r0);
        m1[r] = ld(b.met + (r * 3 + 1) * V + r1);
        m2[r] = ld(b.met + (r * 3 + 2) * V + r2);
      }
#pragma unroll
      for (int c = 3; c < 9; ++c) {
        const T *Fc = F + c * V;
        const T g0 = b.ubw[0][k] * ld(Fc + r0), g1 = b.ubw[1][k] * ld(Fc + r1), g2 = b.ubw[2][k] * ld(Fc + r2);
        DFx[c] = DFx[c] + g0 * m0[0] * J0 + g1 * m1[0] * J1 + g2 * m2[0] * J2;
        DFy[c] = DFy[c] + g0 * m0[1] * J0 + g1 * m1[1] * J1 + g2 * m2[1] * J2;
        DFz[c] = DFz[c] + g0 * m0[2] * J0 + g1 * m1[2] * J1 + g2 * m2[2] * J2;
      }
    }
  }
}

// Separable Cartesian near-boundary derivative of all nine fields along one
// axis: m_a(i) * (1/h_a) * sum_k c_k F(k).  On a Cartesian grid whose metric
// is diagonal to roundoff, J*X_a is constant along the axis, so this equals
// JJU_x6's conservative form divided by J (src/JU_xJU_yJU_z6.f90:12-809).
template <typename T>
__device__ void sep_axis(const Blk<T> &b, const T *F, int a, int i, int n, long long p, long long stride, T m, T ih,
                         T U[9]) {
  T s[9];
#pragma unroll
  for (int f = 0; f < 9; ++f) s[f] = 0;
  if (central_row(b, a, i, n)) {
    const T cc[6] = {(T)(-1.0 / 60.0), (T)0.15, (T)-0.75, (T)0.75, (T)-0.15, (T)(1.0 / 60.0)};
    const int off[6] = {-3, -2, -1, 1, 2, 3};
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const long long q = p + (long long)off[k] * stride;
#pragma unroll
      for (int f = 0; f < 9; ++f) s[f] = s[f] + cc[k] * ld(F + f * b.vol + q);
    }
  } else {
    const int row = i <= 6 ? i - 1 : 6 + (n - i);
    const double *rc = b.rowc + row * 8;
    const int *ro = b.rowo + row * 8;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const T c = (T)__ldg(rc + k);
      if (c != (T)0) {
        const long long q = p + (long long)__ldg(ro + k) * stride;
#pragma unroll
        for (int f = 0; f < 9; ++f) s[f] = s[f] + c * ld(F + f * b.vol + q);
      }
    }
  }
#pragma unroll
  for (int f = 0; f < 9; ++f) U[f] = ih * (m * s[f]);
}

// ---------------------------------------------------------------------------
// Stage kernel: one thread per grid point.
// ---------------------------------------------------------------------------
// the lean memory-variable update (defined with the curvilinear passes)
template <typename T, int RESP, int C0 = 0, int C1 = 6>
__device__ __forceinline__ void anelastic_lean(const Blk<T> &b, const StageArgs &a, int x, int y, int z, long long p, T lam,
                                               T mu, const T e[6], T tr, T s[9], bool do_rhs);

// LEAN: memory variables through anelastic_lean (per-point factors, 1/tau
// multiplied; the Cartesian shell) instead of anelastic_point's reference
// association
template <typename T, int MESH, int RESP, bool SEP = false, bool GIN = false, bool LEAN = false>
__device__ void point_update(const Blk<T> &b, const StageArgs &a, int x, int y, int z) {
  const long long p = pidx(b, x, y, z);
  const long long V = b.vol;
  const T *F = a.cur ? b.F1 : b.F0;
  T *Fn = a.cur ? b.F0 : b.F1;
  if (a.flags & F_UPDATE) {
    // F and the compensation are read by the update at the end
#pragma unroll
    for (int c = 0; c < 9; ++c) prefetch_l2(F + c * V + p);
    if (b.FC) {
#pragma unroll
      for (int c = 0; c < 9; ++c) prefetch_l2(b.FC + c * V + p);
    }
  }
  const double t0 = a.time ? a.time->t : 0.0;
  const double tst = a.stage <= 1 ? t0 : t0 + c_rkC[a.stage - 1] * a.dt;

  T df[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    T v = b.DF[c * V + p];
    df[c] = (a.flags & F_SCALE) ? (T)a.A * v : v;
  }
  const bool interior = x >= b.lo[0] && x <= b.hi[0] && y >= b.lo[1] && y <= b.hi[1] && z >= b.lo[2] && z <= b.hi[2];
  bool in_pml = false;
  if (b.npml > 0) {
    for (int f = 0; f < 6; ++f) {
      if (!b.pml_on[f]) continue;
      const int *B = b.pb[f];
      if (x >= B[0] && x <= B[1] && y >= B[2] && y <= B[3] && z >= B[4] && z <= B[5]) in_pml = true;
    }
  }
  // scale / integrate PML rates of points not reached by the RHS path
  const bool rhs = (a.flags & F_RHS) != 0;

  if (rhs && interior && !GIN) {
    // strict interior, src/JU_xJU_yJU_z6.f90:16177-16636
    T DFx[9], DFy[9], DFz[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) { DFx[c] = 0; DFy[c] = 0; DFz[c] = 0; }
    if (b.fd != 0) {
      up_interior<T, MESH>(b, F, x, y, z, p, DFx, DFy, DFz);
    } else if (MESH == MESH_CART) {
      const T mx = ld(b.mq + x), my = ld(b.mr + y), mz = ld(b.ms + z);
#pragma unroll
      for (int s = 1; s <= 3; ++s) {
        const T ax = mx * b.cx[s - 1], ay = my * b.cy[s - 1], az = mz * b.cz[s - 1];
#pragma unroll
        for (int c = 0; c < 9; ++c) {
          const T *Fc = F + c * V;
          DFx[c] = DFx[c] + ax * (ld(Fc + p + s) - ld(Fc + p - s));
          DFy[c] = DFy[c] + ay * (ld(Fc + p + s * b.sy) - ld(Fc + p - s * b.sy));
          DFz[c] = DFz[c] + az * (ld(Fc + p + s * b.sz) - ld(Fc + p - s * b.sz));
        }
      }
    } else {
      const T *met = b.met;
      T mp[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) mp[k] = ld(met + k * V + p);
#pragma unroll
      for (int s = 1; s <= 3; ++s) {
        const long long off[3] = {s, s * b.sy, s * b.sz};
        const T cc[3] = {b.cx[s - 1], b.cy[s - 1], b.cz[s - 1]};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const T *Fc = F + c * V;
          T d0 = ld(Fc + p + off[0]) - ld(Fc + p - off[0]);
          T d1 = ld(Fc + p + off[1]) - ld(Fc + p - off[1]);
          T d2 = ld(Fc + p + off[2]) - ld(Fc + p - off[2]);
          DFx[c] = DFx[c] + mp[0] * cc[0] * d0 + mp[1] * cc[1] * d1 + mp[2] * cc[2] * d2;
          DFy[c] = DFy[c] + mp[3] * cc[0] * d0 + mp[4] * cc[1] * d1 + mp[5] * cc[2] * d2;
          DFz[c] = DFz[c] + mp[6] * cc[0] * d0 + mp[7] * cc[1] * d1 + mp[8] * cc[2] * d2;
        }
        // conservative stress derivatives, J * metric at the neighbours
        T jm[3][3][2];  // [row][axis][+/-]
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
          long long qp_ = p + off[ax], qm_ = p - off[ax];
          T Jp = ld(b.J + qp_), Jm = ld(b.J + qm_);
#pragma unroll
          for (int row = 0; row < 3; ++row) {
            jm[row][ax][0] = Jp * ld(met + (row * 3 + ax) * V + qp_);
            jm[row][ax][1] = Jm * ld(met + (row * 3 + ax) * V + qm_);
          }
        }
#pragma unroll
        for (int c = 3; c < 9; ++c) {
          const T *Fc = F + c * V;
          T fp0 = ld(Fc + p + off[0]), fm0 = ld(Fc + p - off[0]);
          T fp1 = ld(Fc + p + off[1]), fm1 = ld(Fc + p - off[1]);
          T fp2 = ld(Fc + p + off[2]), fm2 = ld(Fc + p - off[2]);
          DFx[c] = DFx[c] + cc[0] * (fp0 * jm[0][0][0] - fm0 * jm[0][0][1]) + cc[1] * (fp1 * jm[0][1][0] - fm1 * jm[0][1][1]) +
                   cc[2] * (fp2 * jm[0][2][0] - fm2 * jm[0][2][1]);
          DFy[c] = DFy[c] + cc[0] * (fp0 * jm[1][0][0] - fm0 * jm[1][0][1]) + cc[1] * (fp1 * jm[1][1][0] - fm1 * jm[1][1][1]) +
                   cc[2] * (fp2 * jm[1][2][0] - fm2 * jm[1][2][1]);
          DFz[c] = DFz[c] + cc[0] * (fp0 * jm[2][0][0] - fm0 * jm[2][0][1]) + cc[1] * (fp1 * jm[2][1][0] - fm1 * jm[2][1][1]) +
                   cc[2] * (fp2 * jm[2][2][0] - fm2 * jm[2][2][1]);
        }
      }
    }
    const T lam = b.M[p], mu = b.M[V + p], rho = b.M[2 * V + p];
    const T a1 = MESH == MESH_CART ? (T)1 / rho : (T)1 / (rho * ld(b.J + p));
    const T a2 = (T)2 * mu + lam, a3 = lam, a4 = mu;
    df[0] = df[0] + a1 * (DFx[3] + DFy[6] + DFz[7]);
    df[1] = df[1] + a1 * (DFx[6] + DFy[4] + DFz[8]);
    df[2] = df[2] + a1 * (DFx[7] + DFy[8] + DFz[5]);
    df[3] = df[3] + a2 * DFx[0] + a3 * (DFy[1] + DFz[2]);
    df[4] = df[4] + a2 * DFy[1] + a3 * (DFx[0] + DFz[2]);
    df[5] = df[5] + a2 * DFz[2] + a3 * (DFx[0] + DFy[1]);
    df[6] = df[6] + a4 * (DFy[0] + DFx[1]);
    df[7] = df[7] + a4 * (DFz[0] + DFx[2]);
    df[8] = df[8] + a4 * (DFz[1] + DFy[2]);
    if (RESP != RESP_EL) {
      T e[6] = {DFx[0], DFy[1], DFz[2], DFy[0] + DFx[1], DFz[0] + DFx[2], DFz[1] + DFy[2]};
      T tr = DFx[0] + DFy[1] + DFz[2];
      if constexpr (LEAN) anelastic_lean<T, RESP>(b, a, x, y, z, p, lam, mu, e, tr, df, true);
      else anelastic_point<T, RESP>(b, a, x, y, z, p, e, tr, df, true);
    }
  } else if (rhs) {
    // near boundaries and PML slabs, src/RHS_Interior.f90:136-281
    T Ux[9], Uy[9], Uz[9];
    const T lam = b.M[p], mu = b.M[V + p], rho = b.M[2 * V + p];
    T J, rhoJ_inv;
    if (GIN) {
      // the derivative terms k_curv_grad left for this point
      const T *Gp = b.G + p;
#pragma unroll
      for (int f = 0; f < 3; ++f) {
        Ux[f] = Gp[(0 + f) * V];
        Uy[f] = Gp[(3 + f) * V];
        Uz[f] = Gp[(6 + f) * V];
      }
      Ux[3] = Gp[9 * V];  Ux[6] = Gp[10 * V]; Ux[7] = Gp[11 * V];
      Uy[6] = Gp[12 * V]; Uy[4] = Gp[13 * V]; Uy[8] = Gp[14 * V];
      Uz[7] = Gp[15 * V]; Uz[8] = Gp[16 * V]; Uz[5] = Gp[17 * V];
      Ux[4] = Ux[5] = Ux[8] = (T)0;
      Uy[3] = Uy[5] = Uy[7] = (T)0;
      Uz[3] = Uz[4] = Uz[6] = (T)0;
      J = ld(b.J + p);
      rhoJ_inv = (T)1 / (rho * J);
    } else if (SEP) {
      sep_axis<T>(b, F, 0, x, b.nx, p, 1, ld(b.mq + x), b.ihq, Ux);
      sep_axis<T>(b, F, 1, y, b.ny, p, b.sy, ld(b.mr + y), b.ihr, Uy);
      sep_axis<T>(b, F, 2, z, b.nz, p, b.sz, ld(b.ms + z), b.ihs, Uz);
      J = (T)1;
      rhoJ_inv = (T)1 / rho;
    } else {
      T U[3][9];
      if (b.fd != 0) jju_up_all<T>(b, F, x, y, z, p, U);
      else jju6_all<T>(b, F, x, y, z, p, U);
#pragma unroll
      for (int f = 0; f < 9; ++f) { Ux[f] = U[0][f]; Uy[f] = U[1][f]; Uz[f] = U[2][f]; }
      J = ld(b.J + p);
      rhoJ_inv = (T)1 / (rho * J);
    }
    const T lambda2mu = lam + (T)2 * mu;
    T DU[9];
    DU[0] = (Ux[3] + Uy[6] + Uz[7]) * rhoJ_inv;
    DU[1] = (Ux[6] + Uy[4] + Uz[8]) * rhoJ_inv;
    DU[2] = (Ux[7] + Uy[8] + Uz[5]) * rhoJ_inv;
    DU[3] = lambda2mu * Ux[0] + lam * (Uy[1] + Uz[2]);
    DU[4] = lambda2mu * Uy[1] + lam * (Ux[0] + Uz[2]);
    DU[5] = lambda2mu * Uz[2] + lam * (Ux[0] + Uy[1]);
    DU[6] = mu * (Uy[0] + Ux[1]);
    DU[7] = mu * (Uz[0] + Ux[2]);
    DU[8] = mu * (Uz[1] + Uy[2]);
    if (RESP != RESP_EL) {
      T e[6] = {Ux[0], Uy[1], Uz[2], Uy[0] + Ux[1], Uz[0] + Ux[2], Uz[1] + Uy[2]};
      T tr;
      if (in_pml && pml_strain_correction<T>(b, x, y, z, e)) tr = e[0] + e[1] + e[2];
      else tr = Ux[0] + Uy[1] + Uz[2];
      if constexpr (LEAN) anelastic_lean<T, RESP>(b, a, x, y, z, p, lam, mu, e, tr, DU, true);
      else anelastic_point<T, RESP>(b, a, x, y, z, p, e, tr, DU, true);
    }
    if (in_pml) {
      // scale the slab rates first (scale_rates runs before set_rates)
      if (a.flags & F_SCALE) {
        for (int f = 0; f < 6; ++f) {
          if (!b.pml_on[f]) continue;
          const int *B = b.pb[f];
          if (x < B[0] || x > B[1] || y < B[2] || y > B[3] || z < B[4] || z > B[5]) continue;
          long long q = (long long)(x - B[0]) + (long long)(B[1] - B[0] + 1) * ((long long)(y - B[2]) + (long long)(B[3] - B[2] + 1) * (long long)(z - B[4]));
          for (int c = 0; c < 9; ++c) b.DQ[f][c * b.pvol[f] + q] = (T)a.A * b.DQ[f][c * b.pvol[f] + q];
        }
      }
      pml_point<T, !SEP>(b, a, x, y, z, p, Ux, Uy, Uz, rhoJ_inv, lambda2mu, J, DU);
    }
#pragma unroll
    for (int c = 0; c < 9; ++c) df[c] = df[c] + DU[c];
  } else {
    // no RHS this pass: still scale point-local memory-variable / PML rates
    if (RESP != RESP_EL && (a.flags & (F_SCALE | F_UPDATE))) {
      T e[6] = {0, 0, 0, 0, 0, 0};
      anelastic_point<T, RESP>(b, a, x, y, z, p, e, (T)0, df, false);
    }
    if (in_pml && (a.flags & F_SCALE)) {
      for (int f = 0; f < 6; ++f) {
        if (!b.pml_on[f]) continue;
        const int *B = b.pb[f];
        if (x < B[0] || x > B[1] || y < B[2] || y > B[3] || z < B[4] || z > B[5]) continue;
        long long q = (long long)(x - B[0]) + (long long)(B[1] - B[0] + 1) * ((long long)(y - B[2]) + (long long)(B[3] - B[2] + 1) * (long long)(z - B[4]));
        for (int c = 0; c < 9; ++c) b.DQ[f][c * b.pvol[f] + q] = (T)a.A * b.DQ[f][c * b.pvol[f] + q];
      }
    }
  }

  if ((a.flags & F_SOURCE) && b.nsrc > 0 && x >= b.sbox[0] && x <= b.sbox[1] && y >= b.sbox[2] && y <= b.sbox[3] &&
      z >= b.sbox[4] && z <= b.sbox[5])
    add_sources<T, MESH>(b, tst, x, y, z, p, df);
  if (b.mms && (a.flags & F_SOURCE)) mms_forcing<T>(b, tst, p, df);
  if ((a.flags & F_SAT) && (x == 1 || x == b.nx || y == 1 || y == b.ny || z == 1 || z == b.nz))
    add_face_sats<T, MESH, SEP>(b, F, x, y, z, p, df, in_pml, tst);
  if ((a.flags & F_ISAT)) {
    // interface SAT, src/RHS_Interior.f90:1813-1837: DF(face) -= tau0/hx * (F_x | G_x)
    int side = x == 1 ? 0 : (x == b.nx ? 1 : -1);
    if (side >= 0 && b.isat[side]) {
      const T pen = b.tau0 / b.hq;
      long long fp = (long long)(y - 1) + (long long)b.ny * (z - 1);
      long long fn = (long long)b.ny * b.nz;
#pragma unroll
      for (int c = 0; c < 9; ++c) df[c] = df[c] - pen * b.isat[side][c * fn + fp];
    }
  }
#pragma unroll
  for (int c = 0; c < 9; ++c) b.DF[c * V + p] = df[c];
  if (a.flags & F_UPDATE) {
    const T Bdt = (T)a.Bdt;
    if (b.FC) {
      // FP32: compensated (Kahan) accumulation of F
#pragma unroll
      for (int c = 0; c < 9; ++c) {
        T f0 = F[c * V + p];
        T comp = b.FC[c * V + p];
        T yv = Bdt * df[c] - comp;
        T tv = f0 + yv;
        b.FC[c * V + p] = (tv - f0) - yv;
        Fn[c * V + p] = tv;
      }
    } else {
#pragma unroll
      for (int c = 0; c < 9; ++c) Fn[c * V + p] = F[c * V + p] + Bdt * df[c];
    }
    if (in_pml) {
      for (int f = 0; f < 6; ++f) {
        if (!b.pml_on[f]) continue;
        const int *B = b.pb[f];
        if (x < B[0] || x > B[1] || y < B[2] || y > B[3] || z < B[4] || z > B[5]) continue;
        long long q = (long long)(x - B[0]) + (long long)(B[1] - B[0] + 1) * ((long long)(y - B[2]) + (long long)(B[3] - B[2] + 1) * (long long)(z - B[4]));
        for (int c = 0; c < 9; ++c) b.Q[f][c * b.pvol[f] + q] = b.Q[f][c * b.pvol[f] + q] + Bdt * b.DQ[f][c * b.pvol[f] + q];
      }
    }
  }
}

template <typename T, int MESH, int RESP>
__global__ void __launch_bounds__(256) k_stage(Blk<T> b, StageArgs a) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int y = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int z = blockIdx.z * blockDim.z + threadIdx.z + 1;
  if (x > b.nx || y > b.ny || z > b.nz) return;
  point_update<T, MESH, RESP>(b, a, x, y, z);
}

// ---------------------------------------------------------------------------
// Curvilinear stage, first pass: the derivative terms of JJU_x6
// (src/JU_xJU_yJU_z6.f90:12-809) that the point update uses, for every point
// of the block, interior and near-boundary alike (the reference's interior
// form, src/JU_xJU_yJU_z6.f90:16177-16424, is the same operator with the
// central row, summed in another order).  Per axis a with row coefficients
// c_k: velocities X_r(p) * (1/h_a) sum_k c_k v(k), stresses
// sum_k (s(k) ((c_k / h_a) J(k))) X_r(k) for the nine (stress, metric row)
// pairs the rates need, summed over the three axes in one accumulator each
// (the reference scales each axis sum by 1/h_a: rounding-level difference).  G holds, component-major with the field stride:
//   0-8   dv_x/dx, dv_y/dx, dv_z/dx, dv_x/dy, ..., dv_z/dz   (Ux, Uy, Uz 1:3)
//   9-17  Ux4, Ux7, Ux8, Uy7, Uy5, Uy9, Uz8, Uz9, Uz6        (1-based JJU_x6 slots)
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ bool flat_point(const Blk<T> &b, int &x, int &y, int &z);

// The 18 derivative terms of one point (layout of G above) into registers.
template <typename T>
__device__ __forceinline__ void curv_derivs(const Blk<T> &b, const T *__restrict__ F, int x, int y, int z, long long p,
                                            T U[9], T S[9]) {
  const long long V = b.vol;
  const int pos[3] = {x, y, z};
  const int nn[3] = {b.nx, b.ny, b.nz};
  const long long st[3] = {1, b.sy, b.sz};
  const T ih[3] = {b.ihq, b.ihr, b.ihs};
#pragma unroll
  for (int k = 0; k < 9; ++k) { U[k] = 0; S[k] = 0; }
#pragma unroll 1
  for (int ax = 0; ax < 3; ++ax) {
    T sv[3] = {0, 0, 0};
    const T h = ih[ax];
    const T *X0 = b.met + (long long)(0 * 3 + ax) * V;
    const T *X1 = b.met + (long long)(1 * 3 + ax) * V;
    const T *X2 = b.met + (long long)(2 * 3 + ax) * V;
    // stress fluxes straight into S with 1/h folded into the tap weight (no
    // per-axis accumulators: registers go to loads in flight)
    auto tap = [&](long long q, T c) {
      const T cJ = (h * c) * ld(b.J + q);
      const T x0 = ld(X0 + q), x1 = ld(X1 + q), x2 = ld(X2 + q);
#pragma unroll
      for (int f = 0; f < 3; ++f) sv[f] = sv[f] + c * ld(F + f * V + q);
      const T sxx = ld(F + 3 * V + q) * cJ, syy = ld(F + 4 * V + q) * cJ;
      const T szz = ld(F + 5 * V + q) * cJ, sxy = ld(F + 6 * V + q) * cJ;
      const T sxz = ld(F + 7 * V + q) * cJ, syz = ld(F + 8 * V + q) * cJ;
      S[0] = S[0] + sxx * x0; S[1] = S[1] + sxy * x0; S[2] = S[2] + sxz * x0;
      S[3] = S[3] + sxy * x1; S[4] = S[4] + syy * x1; S[5] = S[5] + syz * x1;
      S[6] = S[6] + sxz * x2; S[7] = S[7] + syz * x2; S[8] = S[8] + szz * x2;
    };
    const int i = pos[ax], n = nn[ax];
    if (central_row(b, ax, i, n)) {
      const T cc[6] = {(T)(-1.0 / 60.0), (T)0.15, (T)-0.75, (T)0.75, (T)-0.15, (T)(1.0 / 60.0)};
      const int off[6] = {-3, -2, -1, 1, 2, 3};
#pragma unroll
      for (int k = 0; k < 6; ++k) tap(p + (long long)off[k] * st[ax], cc[k]);
    } else {
      const int row = i <= 6 ? i - 1 : 6 + (n - i);
      const double *rc = b.rowc + row * 8;
      const int *ro = b.rowo + row * 8;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const T c = (T)__ldg(rc + k);
        if (c != (T)0) tap(p + (long long)__ldg(ro + k) * st[ax], c);
      }
    }
    const T xp[3] = {ld(X0 + p), ld(X1 + p), ld(X2 + p)};
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int f = 0; f < 3; ++f) U[r * 3 + f] = U[r * 3 + f] + h * (xp[r] * sv[f]);
  }
}

// FLAT: one thread per point of a flattened (x fastest) 1-D launch, every lane
// busy; otherwise 3-D tiles of blockDim points.
template <typename T, int MINB, int FLAT>
__global__ void __launch_bounds__(256, MINB) k_curv_grad(Blk<T> b, int cur) {
  int x, y, z;
  if (FLAT) {
    if (!flat_point(b, x, y, z)) return;
  } else {
    x = blockIdx.x * blockDim.x + threadIdx.x + 1;
    y = blockIdx.y * blockDim.y + threadIdx.y + 1;
    z = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (x > b.nx || y > b.ny || z > b.nz) return;
  }
  const long long p = pidx(b, x, y, z);
  const long long V = b.vol;
  T U[9], S[9];
  curv_derivs<T>(b, cur ? b.F1 : b.F0, x, y, z, p, U, S);
  T *Gp = b.G + p;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    Gp[k * V] = U[k];
    Gp[(9 + k) * V] = S[k];
  }
}

// Curvilinear stage, second pass: every point through the near-boundary
// point update with the derivative terms of k_curv_grad (anelastic, PML,
// sources, SATs, interface SAT, RK update).
template <typename T, int RESP>
__global__ void __launch_bounds__(256, 2) k_curv_update(Blk<T> b, StageArgs a) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int y = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int z = blockIdx.z * blockDim.z + threadIdx.z + 1;
  if (x > b.nx || y > b.ny || z > b.nz) return;
  point_update<T, MESH_CURV, RESP, false, true>(b, a, x, y, z);
}

// ---------------------------------------------------------------------------
// Lean curvilinear point update (the second pass after k_curv_grad): the
// near-boundary point update of src/RHS_Interior.f90:136-281 for every point
// -- rates from the derivative terms, memory variables
// (src/RHS_Interior.f90:2599-2908, :3361-3477), PML with the anelastic strain
// correction (:1846-2265, :2351-2451), sources, face and interface SATs and
// the RK update -- written for memory-level parallelism:
//   * the six PML slabs are visited with compile-time face indices, so the
//     slab boxes, damping and Q / DQ stay in registers; Q and DQ are read
//     once and written once per stage (scale, source, integrate);
//   * memory variables are streamed through restrict pointers so the loads
//     of the next component can be issued before the stores of this one;
//   * 1/tau is applied as a multiplication (one rounding instead of a
//     division; well inside the parity tolerance).
// ---------------------------------------------------------------------------
template <typename T, int F>
__device__ __forceinline__ bool slab_has(const Blk<T> &b, int x, int y, int z) {
  if (!b.pml_on[F]) return false;
  const int *B = b.pb[F];
  return x >= B[0] && x <= B[1] && y >= B[2] && y <= B[3] && z >= B[4] && z <= B[5];
}

template <typename T, int F>
__device__ __forceinline__ long long slab_index(const Blk<T> &b, int x, int y, int z) {
  const int *B = b.pb[F];
  return (long long)(x - B[0]) + (long long)(B[1] - B[0] + 1) * ((long long)(y - B[2]) + (long long)(B[3] - B[2] + 1) * (long long)(z - B[4]));
}

template <typename T, int F>
__device__ __forceinline__ T slab_damping(const Blk<T> &b, int x, int y, int z) {
  constexpr int axis = F >> 1;
  const int i = axis == 0 ? x : axis == 1 ? y : z;
  const int n = axis == 0 ? b.nx : axis == 1 ? b.ny : b.nz;
  const T v = (F == 4) ? (T)(i - b.npml) : ((F & 1) ? (T)(i - (n - b.npml)) : (T)(i - (1 + b.npml)));
  return b.d0 * fabs(v / (T)b.npml);
}

// face-local index of (x, y, z) on face F
template <typename T, int F>
__device__ __forceinline__ int face_index(const Blk<T> &b, int x, int y, int z) {
  constexpr int axis = F >> 1;
  return axis == 0 ? (y - 1) + b.ny * (z - 1) : axis == 1 ? (x - 1) + b.nx * (z - 1) : (x - 1) + b.nx * (y - 1);
}

template <typename T, int F>
__device__ __forceinline__ bool on_face(const Blk<T> &b, int x, int y, int z) {
  constexpr int axis = F >> 1;
  const int i = axis == 0 ? x : axis == 1 ? y : z;
  const int n = axis == 0 ? b.nx : axis == 1 ? b.ny : b.nz;
  return (F & 1) ? i == n : i == 1;
}

// One PML slab per axis: the point lies in at most one of the axis's two
// slabs (the host sends blocks whose two slabs on an axis overlap to the
// generic update).  Only the membership is kept; the slab index, damping and
// array pointers are recomputed where they are used.
struct AxisSlab {
  bool lo, hi;
  __device__ __forceinline__ bool in() const { return lo || hi; }
};

template <typename T, int AX>
__device__ __forceinline__ AxisSlab axis_slab(const Blk<T> &b, int x, int y, int z) {
  AxisSlab s;
  s.hi = slab_has<T, 2 * AX + 1>(b, x, y, z);
  s.lo = !s.hi && slab_has<T, 2 * AX>(b, x, y, z);
  return s;
}

// L2 prefetch of the slab-local Q and DQ of this point on one axis (read
// late, after the rates, by slab_do)
template <typename T, int AX>
__device__ __forceinline__ void slab_prefetch(const Blk<T> &b, int x, int y, int z, AxisSlab s) {
  if (!s.in()) return;
  constexpr int FL = 2 * AX, FH = 2 * AX + 1;
  const long long q = s.hi ? slab_index<T, FH>(b, x, y, z) : slab_index<T, FL>(b, x, y, z);
  const long long PV = s.hi ? b.pvol[FH] : b.pvol[FL];
  const T *Qp = (s.hi ? b.Q[FH] : b.Q[FL]) + q;
  const T *DQp = (s.hi ? b.DQ[FH] : b.DQ[FL]) + q;
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    prefetch_l2(Qp + c * PV);
    prefetch_l2(DQp + c * PV);
  }
}

// one slab F of one point: scale DQ (F_SCALE), subtract the PML damping terms
// from the rates and add the auxiliary-field sources to DQ (rhs;
// src/RHS_Interior.f90:1913-2265, J form; the source terms are re-read from
// the derivative scratch Gp), store DQ and integrate Q (integrate)
// derivative terms of one point (G slot k): from the scratch G ...
template <typename T>
struct GMem {
  const T *p;
  long long V;
  __device__ __forceinline__ T operator()(int k) const { return p[k * V]; }
};
// ... or from registers (the fused stage kernel)
template <typename T>
struct GReg {
  const T *U, *S;
  __device__ __forceinline__ T operator()(int k) const { return k < 9 ? U[k] : S[k - 9]; }
};

template <typename T, int F, typename GA>
__device__ __forceinline__ void slab_do(const Blk<T> &b, const StageArgs &a, int x, int y, int z, bool rhs,
                                        bool integrate, bool sat, const GA &G, T rhoJ_inv,
                                        T lambda2mu, T lam, T mu, T J, T df[9]) {
  constexpr int AX = F >> 1;
  const long long q = slab_index<T, F>(b, x, y, z);
  const long long PV = b.pvol[F];
  T *Qp = b.Q[F] + q;
  T *DQp = b.DQ[F] + q;
  T Q[9], DQ[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    Q[c] = Qp[c * PV];
    const T v = DQp[c * PV];
    DQ[c] = (a.flags & F_SCALE) ? (T)a.A * v : v;
  }
  if (rhs) {
    const T d = slab_damping<T, F>(b, x, y, z);
    df[0] = df[0] - d * J * Q[0] * rhoJ_inv;
    df[1] = df[1] - d * J * Q[1] * rhoJ_inv;
    df[2] = df[2] - d * J * Q[2] * rhoJ_inv;
    df[3] = df[3] - d * (lambda2mu * Q[3] + lam * Q[4] + lam * Q[5]);
    df[4] = df[4] - d * (lam * Q[3] + lambda2mu * Q[4] + lam * Q[5]);
    df[5] = df[5] - d * (lam * Q[3] + lam * Q[4] + lambda2mu * Q[5]);
    df[6] = df[6] - mu * d * Q[6];
    df[7] = df[7] - mu * d * Q[7];
    df[8] = df[8] - mu * d * Q[8];
    // G slots: 0-8 velocity gradients (Ux, Uy, Uz 1:3), 9-17 Ux4 Ux7 Ux8 Uy7 Uy5 Uy9 Uz8 Uz9 Uz6
    T src[9];
    if (AX == 2) {
      src[0] = G(15) / J; src[1] = G(16) / J; src[2] = G(17) / J; src[3] = 0; src[4] = 0;
      src[5] = G(8); src[6] = 0; src[7] = G(6); src[8] = G(7);
    } else if (AX == 1) {
      src[0] = G(12) / J; src[1] = G(13) / J; src[2] = G(14) / J; src[3] = 0; src[4] = G(4);
      src[5] = 0; src[6] = G(3); src[7] = 0; src[8] = G(5);
    } else {
      src[0] = G(9) / J; src[1] = G(10) / J; src[2] = G(11) / J; src[3] = G(0); src[4] = 0;
      src[5] = 0; src[6] = G(1); src[7] = G(2); src[8] = 0;
    }
    const T cfs = (T)1;
#pragma unroll
    for (int c = 0; c < 9; ++c) DQ[c] = DQ[c] + src[c] - (d + cfs) * Q[c];
  }
  if (sat && b.fdq[F] && on_face<T, F>(b, x, y, z)) {
    // the face SAT's share of this slab (impose_boundary_condition, PML DQ)
    const int fn = b.foff[F + 1] - b.foff[F];
    const T *q = b.fdq[F] + face_index<T, F>(b, x, y, z);
#pragma unroll
    for (int c = 0; c < 9; ++c) DQ[c] = DQ[c] - q[c * fn];
  }
  const T Bdt = (T)a.Bdt;
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    DQp[c * PV] = DQ[c];
    if (integrate) Qp[c * PV] = Q[c] + Bdt * DQ[c];
  }
}

template <typename T, int AX, typename GA>
__device__ __forceinline__ void slab_pass(const Blk<T> &b, const StageArgs &a, int x, int y, int z, AxisSlab s,
                                          bool rhs, bool integrate, bool sat, const GA &G, T rhoJ_inv,
                                          T lambda2mu, T lam, T mu, T J, T df[9]) {
  if (s.hi) slab_do<T, 2 * AX + 1>(b, a, x, y, z, rhs, integrate, sat, G, rhoJ_inv, lambda2mu, lam, mu, J, df);
  else if (s.lo) slab_do<T, 2 * AX>(b, a, x, y, z, rhs, integrate, sat, G, rhoJ_inv, lambda2mu, lam, mu, J, df);
}

// PML strain correction term d * Q[c] of the slab of one axis (0 outside)
template <typename T, int AX>
__device__ __forceinline__ void slab_strain(const Blk<T> &b, int x, int y, int z, AxisSlab s, int c0, int c1, int c2,
                                            T &d, T &q0, T &q1, T &q2) {
  d = 0; q0 = 0; q1 = 0; q2 = 0;
  if (!s.in()) return;
  constexpr int FL = 2 * AX, FH = 2 * AX + 1;
  const long long q = s.hi ? slab_index<T, FH>(b, x, y, z) : slab_index<T, FL>(b, x, y, z);
  const long long PV = s.hi ? b.pvol[FH] : b.pvol[FL];
  const T *Qp = (s.hi ? b.Q[FH] : b.Q[FL]) + q;
  d = s.hi ? slab_damping<T, FH>(b, x, y, z) : slab_damping<T, FL>(b, x, y, z);
  q0 = Qp[c0 * PV]; q1 = Qp[c1 * PV]; q2 = Qp[c2 * PV];
}

// Rates and update of the N memory variables of stress component c at one
// point: ev / dv hold eta and deta on entry, the values to store on return;
// the sum of the old eta is subtracted from the stress rate s[3 + c] (when
// do_rhs), the rates scaled / accumulated, eta integrated (F_UPDATE).  The
// rate of src/RHS_Interior.f90:2599-2908 (Q4 / Q8) is regrouped per component
// as w_l * (2 mu Qs^-1 e) + w_l * (((lambda + 2 mu) Qp^-1 - 2 mu Qs^-1) tr)
// and that of :3361-3477 (fQ8) as s_l (2 mu e) + (p_l (lambda + 2 mu) tr -
// s_l 2 mu tr), so only per-point scalars and the per-mechanism constants
// are live: the same products in another association (rounding level).
template <typename T, int RESP, int N>
__device__ __forceinline__ void mv_component(const Blk<T> &b, const StageArgs &a, int c, int active, T fn, T ft, T fs,
                                             T l2m, T two_mu, const T e[6], T tr, T s[9], bool do_rhs, T ev[N],
                                             T dv[N]) {
  const T A = (T)a.A, Bdt = (T)a.Bdt;
#pragma unroll
  for (int i = 0; i < N; ++i)
    if (a.flags & F_SCALE) dv[i] = A * dv[i];
  if (do_rhs) {
    T sum = ev[0];
#pragma unroll
    for (int i = 1; i < N; ++i) sum = sum + ev[i];
    s[3 + c] = s[3 + c] - sum;
    const T ge = (c < 3 ? fn : fs) * e[c];
    const T gt = ft * tr, l2t = l2m * tr, m2t = two_mu * tr;
#pragma unroll
    for (int i = 0; i < N; ++i) {
      if (RESP == RESP_FQ8) {
        if (b.coarse && (i + 1) != active) continue;
        const T ss = b.ss[i], ps = b.ps[i];
        if (c < 3) dv[i] = dv[i] + ((ss * ge + (ps * l2t - ss * m2t)) - ev[i]) * b.itau[i];
        else dv[i] = dv[i] + (ss * ge - ev[i]) * b.itau[i];
      } else {
        const T w = b.w[i];
        if (c < 3) dv[i] = dv[i] + ((w * ge + w * gt) - ev[i]) * b.itau[i];
        else dv[i] = dv[i] + (w * ge - ev[i]) * b.itau[i];
      }
    }
  }
  if (a.flags & F_UPDATE) {
#pragma unroll
    for (int i = 0; i < N; ++i) ev[i] = ev[i] + Bdt * dv[i];
  }
}

// per-point factors of the memory-variable rates
template <typename T, int RESP>
__device__ __forceinline__ void mv_factors(const Blk<T> &b, long long p, T lam, T mu, T &fn, T &ft, T &fs, T &l2m,
                                           T &two_mu) {
  T qs = 0, qp = 0;
  if (RESP != RESP_FQ8) { qs = ld(b.qs + p); qp = ld(b.qp + p); }
  two_mu = (T)2 * mu;
  l2m = lam + (T)2 * mu;
  fn = RESP == RESP_FQ8 ? two_mu : two_mu * qs;               // normal strain factor
  ft = RESP == RESP_FQ8 ? (T)0 : (l2m * qp - two_mu * qs);    // trace factor (Q4/Q8)
  fs = RESP == RESP_FQ8 ? mu : mu * qs;                        // shear strain factor
}

// memory variables of one point (stress components C0 .. C1 - 1), straight
// from and to global memory
template <typename T, int RESP, int C0, int C1>
__device__ __forceinline__ void anelastic_lean(const Blk<T> &b, const StageArgs &a, int x, int y, int z, long long p, T lam,
                                               T mu, const T e[6], T tr, T s[9], bool do_rhs) {
  constexpr int N = RESP == RESP_Q4 ? 4 : 8;
  const long long V = b.vol;
  const int active = 1 + ((x - 1) & 1) + 2 * ((y - 1) & 1) + 4 * ((z - 1) & 1);
  T *__restrict__ ep = b.eta + p;
  T *__restrict__ dp = b.deta + p;
  T fn, ft, fs, l2m, two_mu;
  mv_factors<T, RESP>(b, p, lam, mu, fn, ft, fs, l2m, two_mu);
  // the interior tile's half (three components) of an 8-mechanism block one
  // component at a time (fewer registers live beside the tile's z-queues:
  // measured 18 % faster on the fQ8 planar blocks); all else unrolled
#pragma unroll (C1 - C0 == 3 && N == 8 ? 1 : 6)
  for (int c = C0; c < C1; ++c) {
    T ev[N], dv[N];
#pragma unroll
    for (int i = 0; i < N; ++i) {
      ev[i] = ep[(long long)(c * N + i) * V];
      dv[i] = dp[(long long)(c * N + i) * V];
    }
    mv_component<T, RESP, N>(b, a, c, active, fn, ft, fs, l2m, two_mu, e, tr, s, do_rhs, ev, dv);
#pragma unroll
    for (int i = 0; i < N; ++i) {
      dp[(long long)(c * N + i) * V] = dv[i];
      if (a.flags & F_UPDATE) ep[(long long)(c * N + i) * V] = ev[i];
    }
  }
}

// Curvilinear memory variables, a streaming pass between k_curv_grad and
// k_curv_point: strain rates from the velocity gradients of G (PML-corrected
// in slabs), memory-variable rates scaled / accumulated, the per-component
// sums of the memory variables (before this stage's update) left in S6 for
// k_curv_point to subtract from the stress rates, and (F_UPDATE) eta
// integrated.
// point of a flattened (x fastest) 1-D launch over the block; false past the end
template <typename T>
__device__ __forceinline__ bool flat_point(const Blk<T> &b, int &x, int &y, int &z) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= b.nx * b.ny * b.nz) return false;
  const int r = j / b.nx;
  x = j - r * b.nx + 1;
  z = r / b.ny;
  y = r - z * b.ny + 1;
  z = z + 1;
  return true;
}

template <typename T, int RESP, int MINB>
__global__ void __launch_bounds__(128, MINB) k_curv_anelastic(Blk<T> b, StageArgs a) {
  int x, y, z;
  if (!flat_point(b, x, y, z)) return;
  const long long p = pidx(b, x, y, z);
  const long long V = b.vol;
  const bool rhs = (a.flags & F_RHS) != 0;
  const T lam = b.M[p], mu = b.M[V + p];
  T e[6] = {0, 0, 0, 0, 0, 0}, tr = 0;
  if (rhs) {
    const T *Gp = b.G + p;
    const T Ux0 = Gp[0], Ux1 = Gp[V], Ux2 = Gp[2 * V];
    const T Uy0 = Gp[3 * V], Uy1 = Gp[4 * V], Uy2 = Gp[5 * V];
    const T Uz0 = Gp[6 * V], Uz1 = Gp[7 * V], Uz2 = Gp[8 * V];
    e[0] = Ux0; e[1] = Uy1; e[2] = Uz2;
    e[3] = Uy0 + Ux1; e[4] = Uz0 + Ux2; e[5] = Uz1 + Uy2;
    AxisSlab sx = {false, false}, sy = {false, false}, sz = {false, false};
    if (b.npml > 0) {
      sx = axis_slab<T, 0>(b, x, y, z);
      sy = axis_slab<T, 1>(b, x, y, z);
      sz = axis_slab<T, 2>(b, x, y, z);
    }
    if (sx.in() || sy.in() || sz.in()) {
      // src/RHS_Interior.f90:2351-2451
      T dx, qx3, qx6, qx7, dy, qy4, qy6, qy8, dz, qz5, qz7, qz8;
      slab_strain<T, 0>(b, x, y, z, sx, 3, 6, 7, dx, qx3, qx6, qx7);
      slab_strain<T, 1>(b, x, y, z, sy, 4, 6, 8, dy, qy4, qy6, qy8);
      slab_strain<T, 2>(b, x, y, z, sz, 5, 7, 8, dz, qz5, qz7, qz8);
      e[0] = e[0] - dx * qx3;
      e[1] = e[1] - dy * qy4;
      e[2] = e[2] - dz * qz5;
      e[3] = e[3] - dx * qx6 - dy * qy6;
      e[4] = e[4] - dx * qx7 - dz * qz7;
      e[5] = e[5] - dy * qy8 - dz * qz8;
      tr = e[0] + e[1] + e[2];
    } else {
      tr = Ux0 + Uy1 + Uz2;
    }
  }
  T s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  anelastic_lean<T, RESP>(b, a, x, y, z, p, lam, mu, e, tr, s, rhs);
  if (rhs) {
    // s[3 + c] = -sum_l eta_c,l
#pragma unroll
    for (int c = 0; c < 6; ++c) b.S6[c * V + p] = s[3 + c];
  }
}

// Ghost planes of an s-slab (src/mpi3dcomm.f90:459-528): pack the 3 planes
// next to each open face into buf (lower face first; each face ncomp x 3 x
// ny x nx, x fastest), or unpack buf into the 3 ghost planes beyond each open
// face.  Components c < n0 live at a0 + c * vol, the rest at a1.
template <typename T>
__global__ void k_halo(Blk<T> b, T *buf, T *a0, int n0, T *a1, int ncomp, int unpack) {
  const long long plane = (long long)b.nx * b.ny;
  const long long face = (long long)ncomp * 3 * plane;
  const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (j >= 2 * face) return;
  const int hi = j >= face;
  if (hi ? !b.open_hi[2] : !b.open_lo[2]) return;
  long long r = j - hi * face;
  const int c = (int)(r / (3 * plane));
  r -= (long long)c * 3 * plane;
  const int k = (int)(r / plane);
  r -= (long long)k * plane;
  const int y = (int)(r / b.nx) + 1;
  const int x = (int)(r - (long long)(y - 1) * b.nx) + 1;
  const int z = unpack ? (hi ? b.nz + 1 + k : k - 2) : (hi ? b.nz - 2 + k : 1 + k);
  T *a = c < n0 ? a0 + (long long)c * b.vol : a1 + (long long)(c - n0) * b.vol;
  const long long p = pidx(b, x, y, z);
  if (unpack) a[p] = buf[j];
  else buf[j] = a[p];
}

// Face SATs of the curvilinear lean path (impose_boundary_condition,
// src/RHS_Interior.f90:1584-1768, with BC_* and BCm/BCp of
// src/BoundaryConditions.f90): one thread per point of every face with a
// physical boundary condition; the terms the reference subtracts are stored
// face-locally and k_curv_point subtracts them in the reference's face order.
template <typename T>
__global__ void __launch_bounds__(128) k_curv_face_sat(Blk<T> b, int cur) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= b.foff[6]) return;
  int f = 0;
#pragma unroll
  for (int g = 1; g < 6; ++g)
    if (j >= b.foff[g]) f = g;
  const int k = j - b.foff[f];
  const int axis = f >> 1, plus = f & 1;
  const int d0 = axis == 0 ? b.ny : b.nx;
  const int a1 = k / d0, a0 = k - a1 * d0;
  const int fixed = plus ? (axis == 0 ? b.nx : axis == 1 ? b.ny : b.nz) : 1;
  int x, y, z;
  if (axis == 0) { x = fixed; y = a0 + 1; z = a1 + 1; }
  else if (axis == 1) { x = a0 + 1; y = fixed; z = a1 + 1; }
  else { x = a0 + 1; y = a1 + 1; z = fixed; }
  const long long p = pidx(b, x, y, z);
  const T *F = cur ? b.F1 : b.F0;
  T u[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) u[c] = F[c * b.vol + p];
  const T lam = b.M[p], mu = b.M[b.vol + p], rho = b.M[2 * b.vol + p];
  const int type = b.bc[f];
  const T r = type == 1 ? (T)0 : type == 2 ? (T)1 : (T)-1;
  const T c_p = sqrt(((T)2 * mu + lam) / rho);
  const T c_s = sqrt(mu / rho);
  const T Zp = rho * c_p, Zs = rho * c_s;
  const T qx = ld(b.met + (long long)(0 + axis) * b.vol + p);
  const T qy = ld(b.met + (long long)(3 + axis) * b.vol + p);
  const T qz = ld(b.met + (long long)(6 + axis) * b.vol + p);
  const T norm = sqrt(qx * qx + qy * qy + qz * qz);
  const int fn = b.foff[f + 1] - b.foff[f];
  const T *B = b.nrm[f];
  T l[3], m[3], n[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    l[c] = ld(B + (0 + c) * fn + k);
    m[c] = ld(B + (3 + c) * fn + k);
    n[c] = ld(B + (6 + c) * fn + k);
  }
  T ubc[9], Ux[9];
  bc_vector<T>(plus, u, Zs, Zp, r, l, m, n, norm, ubc);
  // structure(), src/RHS_Interior.f90:2267-2287
  const T irho = (T)1 / rho;
  Ux[0] = irho * ubc[0];
  Ux[1] = irho * ubc[1];
  Ux[2] = irho * ubc[2];
  Ux[3] = ((T)2 * mu + lam) * ubc[3] + lam * (ubc[4] + ubc[5]);
  Ux[4] = ((T)2 * mu + lam) * ubc[4] + lam * (ubc[3] + ubc[5]);
  Ux[5] = ((T)2 * mu + lam) * ubc[5] + lam * (ubc[3] + ubc[4]);
  Ux[6] = mu * ubc[6];
  Ux[7] = mu * ubc[7];
  Ux[8] = mu * ubc[8];
  const T h = axis == 0 ? b.hq : axis == 1 ? b.hr : b.hs;
  const T pen = b.tau0 / h;
  T *o = b.fsat[f] + k;
#pragma unroll
  for (int c = 0; c < 9; ++c) o[c * fn] = pen * Ux[c];
  if (b.fdq[f]) {
    T *q = b.fdq[f] + k;
#pragma unroll
    for (int c = 0; c < 9; ++c) q[c * fn] = pen * ubc[c];
  }
}

template <typename T, int F>
__device__ __forceinline__ void face_sat_add(const Blk<T> &b, int x, int y, int z, T df[9]) {
  if (!b.fsat[F] || !on_face<T, F>(b, x, y, z)) return;
  const int fn = b.foff[F + 1] - b.foff[F];
  const T *o = b.fsat[F] + face_index<T, F>(b, x, y, z);
#pragma unroll
  for (int c = 0; c < 9; ++c) df[c] = df[c] - o[c * fn];
}

template <typename T, int RESP, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB) k_curv_point(Blk<T> b, StageArgs a) {
  int x, y, z;
  if (!flat_point(b, x, y, z)) return;
  const long long p = pidx(b, x, y, z);
  const long long V = b.vol;
  const T *__restrict__ F = a.cur ? b.F1 : b.F0;
  T *__restrict__ Fn = a.cur ? b.F0 : b.F1;
  T *__restrict__ DFp = b.DF + p;
  if (a.flags & F_UPDATE) {
    // F and the compensation are read only by the update at the end
#pragma unroll
    for (int c = 0; c < 9; ++c) prefetch_l2(F + c * V + p);
    if (b.FC) {
#pragma unroll
      for (int c = 0; c < 9; ++c) prefetch_l2(b.FC + c * V + p);
    }
  }
  T df[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    const T v = DFp[c * V];
    df[c] = (a.flags & F_SCALE) ? (T)a.A * v : v;
  }
  AxisSlab sx = {false, false}, sy = {false, false}, sz = {false, false};
  if (b.npml > 0) {
    sx = axis_slab<T, 0>(b, x, y, z);
    sy = axis_slab<T, 1>(b, x, y, z);
    sz = axis_slab<T, 2>(b, x, y, z);
  }
  const bool in_pml = sx.in() || sy.in() || sz.in();
  if (in_pml) {
    slab_prefetch<T, 0>(b, x, y, z, sx);
    slab_prefetch<T, 1>(b, x, y, z, sy);
    slab_prefetch<T, 2>(b, x, y, z, sz);
  }
  const bool face_pt = x == 1 || x == b.nx || y == 1 || y == b.ny || z == 1 || z == b.nz;
  const bool integrate = (a.flags & F_UPDATE) != 0;
  const bool sat = (a.flags & F_SAT) != 0;
  const T *Gp = b.G + p;
  const GMem<T> G{Gp, V};
  if (a.flags & F_RHS) {
    const T lam = b.M[p], mu = b.M[V + p], rho = b.M[2 * V + p];
    const T J = ld(b.J + p);
    const T rhoJ_inv = (T)1 / (rho * J);
    const T lambda2mu = lam + (T)2 * mu;
    // rates of src/RHS_Interior.f90:238-254 from the derivative terms
    df[0] = df[0] + (Gp[9 * V] + Gp[12 * V] + Gp[15 * V]) * rhoJ_inv;
    df[1] = df[1] + (Gp[10 * V] + Gp[13 * V] + Gp[16 * V]) * rhoJ_inv;
    df[2] = df[2] + (Gp[11 * V] + Gp[14 * V] + Gp[17 * V]) * rhoJ_inv;
    {
      const T Ux0 = Gp[0], Ux1 = Gp[V], Ux2 = Gp[2 * V];
      const T Uy0 = Gp[3 * V], Uy1 = Gp[4 * V], Uy2 = Gp[5 * V];
      const T Uz0 = Gp[6 * V], Uz1 = Gp[7 * V], Uz2 = Gp[8 * V];
      df[3] = df[3] + (lambda2mu * Ux0 + lam * (Uy1 + Uz2));
      df[4] = df[4] + (lambda2mu * Uy1 + lam * (Ux0 + Uz2));
      df[5] = df[5] + (lambda2mu * Uz2 + lam * (Ux0 + Uy1));
      df[6] = df[6] + mu * (Uy0 + Ux1);
      df[7] = df[7] + mu * (Uz0 + Ux2);
      df[8] = df[8] + mu * (Uz1 + Uy2);
    }
    if (RESP != RESP_EL) {
      // minus the memory-variable sums left by k_curv_anelastic
#pragma unroll
      for (int c = 0; c < 6; ++c) df[3 + c] = df[3 + c] + b.S6[c * V + p];
    }
    // PML damping and auxiliary fields, reference slab order z, y, x
    if (in_pml) {
      slab_pass<T, 2>(b, a, x, y, z, sz, true, integrate, sat, G, rhoJ_inv, lambda2mu, lam, mu, J, df);
      slab_pass<T, 1>(b, a, x, y, z, sy, true, integrate, sat, G, rhoJ_inv, lambda2mu, lam, mu, J, df);
      slab_pass<T, 0>(b, a, x, y, z, sx, true, integrate, sat, G, rhoJ_inv, lambda2mu, lam, mu, J, df);
    }
  } else if (in_pml && (a.flags & (F_SCALE | F_UPDATE | F_SAT))) {
    slab_pass<T, 2>(b, a, x, y, z, sz, false, integrate, sat, G, (T)0, (T)0, (T)0, (T)0, (T)1, df);
    slab_pass<T, 1>(b, a, x, y, z, sy, false, integrate, sat, G, (T)0, (T)0, (T)0, (T)0, (T)1, df);
    slab_pass<T, 0>(b, a, x, y, z, sx, false, integrate, sat, G, (T)0, (T)0, (T)0, (T)0, (T)1, df);
  }
  if ((a.flags & F_SOURCE) && b.nsrc > 0 && x >= b.sbox[0] && x <= b.sbox[1] && y >= b.sbox[2] && y <= b.sbox[3] &&
      z >= b.sbox[4] && z <= b.sbox[5]) {
    const double t0 = a.time ? a.time->t : 0.0;
    const double tst = a.stage <= 1 ? t0 : t0 + c_rkC[a.stage - 1] * a.dt;
    add_sources<T, MESH_CURV>(b, tst, x, y, z, p, df);
  }
  if (sat && face_pt) {
    // face SATs in the reference's order Lx, Rx, Ly, Ry, Lz, Rz
    face_sat_add<T, 0>(b, x, y, z, df);
    face_sat_add<T, 1>(b, x, y, z, df);
    face_sat_add<T, 2>(b, x, y, z, df);
    face_sat_add<T, 3>(b, x, y, z, df);
    face_sat_add<T, 4>(b, x, y, z, df);
    face_sat_add<T, 5>(b, x, y, z, df);
  }
  if (a.flags & F_ISAT) {
    // interface SAT, src/RHS_Interior.f90:1813-1837: DF(face) -= tau0/hx * (F_x | G_x)
    const int side = x == 1 ? 0 : (x == b.nx ? 1 : -1);
    if (side >= 0 && b.isat[side]) {
      const T pen = b.tau0 / b.hq;
      const long long fp = (long long)(y - 1) + (long long)b.ny * (z - 1);
      const long long fn = (long long)b.ny * b.nz;
#pragma unroll
      for (int c = 0; c < 9; ++c) df[c] = df[c] - pen * b.isat[side][c * fn + fp];
    }
  }
#pragma unroll
  for (int c = 0; c < 9; ++c) DFp[c * V] = df[c];
  if (a.flags & F_UPDATE) {
    const T Bdt = (T)a.Bdt;
    if (b.FC) {
#pragma unroll
      for (int c = 0; c < 9; ++c) {
        const T f0 = F[c * V + p];
        const T comp = b.FC[c * V + p];
        const T yv = Bdt * df[c] - comp;
        const T tv = f0 + yv;
        b.FC[c * V + p] = (tv - f0) - yv;
        Fn[c * V + p] = tv;
      }
    } else {
#pragma unroll
      for (int c = 0; c < 9; ++c) Fn[c * V + p] = F[c * V + p] + Bdt * df[c];
    }
  }
}

// ---------------------------------------------------------------------------
// Fused curvilinear stage: the derivative terms of k_curv_grad, the memory
// variables of k_curv_anelastic and the point update of k_curv_point for one
// point per thread of a flattened launch, with the 18 derivative terms and
// the memory-variable sums kept in registers (no scratch G / S6 in HBM).
// Rate terms: A DF + elastic rates, PML damping (slabs z, y, x), minus the
// memory-variable sums, sources, face SATs (from the k_curv_face_sat
// buffers, reference face order), interface SAT; the memory-variable strain
// rates take the PML correction from Q before this stage's Q update, as in
// the split passes.
// ---------------------------------------------------------------------------
template <typename T, int RESP, int MINB>
__global__ void __launch_bounds__(128, MINB) k_curv_fused(Blk<T> b, StageArgs a) {
  int x, y, z;
  if (!flat_point(b, x, y, z)) return;
  const long long p = pidx(b, x, y, z);
  const long long V = b.vol;
  const T *__restrict__ F = a.cur ? b.F1 : b.F0;
  T *__restrict__ Fn = a.cur ? b.F0 : b.F1;
  T *__restrict__ DFp = b.DF + p;
  const bool rhs = (a.flags & F_RHS) != 0;
  const bool integrate = (a.flags & F_UPDATE) != 0;
  const bool sat = (a.flags & F_SAT) != 0;
  if (integrate && b.FC) {
#pragma unroll
    for (int c = 0; c < 9; ++c) prefetch_l2(b.FC + c * V + p);
  }
  if (RESP != RESP_EL && a.pf) {
    // the memory-variable stream is read after the derivative gathers: ask
    // for it now so that its DRAM latency overlaps them
    constexpr int NM = RESP == RESP_Q4 ? 4 : 8;
#pragma unroll 8
    for (int c = 0; c < 6 * NM; ++c) {
      prefetch_l2(b.eta + (long long)c * V + p);
      prefetch_l2(b.deta + (long long)c * V + p);
    }
  }
  AxisSlab sx = {false, false}, sy = {false, false}, sz = {false, false};
  if (b.npml > 0) {
    sx = axis_slab<T, 0>(b, x, y, z);
    sy = axis_slab<T, 1>(b, x, y, z);
    sz = axis_slab<T, 2>(b, x, y, z);
  }
  const bool in_pml = sx.in() || sy.in() || sz.in();
  T U[9], S[9];
  if (rhs) curv_derivs<T>(b, F, x, y, z, p, U, S);
  if (rhs && a.rec) {
    T *E = reinterpret_cast<T *>(a.rec) + p;
    E[0] = U[0]; E[V] = U[4]; E[2 * V] = U[8];
    E[3 * V] = U[3] + U[1]; E[4 * V] = U[6] + U[2]; E[5 * V] = U[7] + U[5];
    E[6 * V] = S[0] + S[3] + S[6]; E[7 * V] = S[1] + S[4] + S[7]; E[8 * V] = S[2] + S[5] + S[8];
  }
  T df[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    const T v = DFp[c * V];
    df[c] = (a.flags & F_SCALE) ? (T)a.A * v : v;
  }
  T lam = 0, mu = 0, J = 1, rhoJ_inv = 0, lambda2mu = 0;
  if (rhs) {
    const T rho = b.M[2 * V + p];
    lam = b.M[p];
    mu = b.M[V + p];
    J = ld(b.J + p);
    rhoJ_inv = (T)1 / (rho * J);
    lambda2mu = lam + (T)2 * mu;
    // rates of src/RHS_Interior.f90:238-254 from the derivative terms
    df[0] = df[0] + (S[0] + S[3] + S[6]) * rhoJ_inv;
    df[1] = df[1] + (S[1] + S[4] + S[7]) * rhoJ_inv;
    df[2] = df[2] + (S[2] + S[5] + S[8]) * rhoJ_inv;
    df[3] = df[3] + (lambda2mu * U[0] + lam * (U[4] + U[8]));
    df[4] = df[4] + (lambda2mu * U[4] + lam * (U[0] + U[8]));
    df[5] = df[5] + (lambda2mu * U[8] + lam * (U[0] + U[4]));
    df[6] = df[6] + mu * (U[3] + U[1]);
    df[7] = df[7] + mu * (U[6] + U[2]);
    df[8] = df[8] + mu * (U[7] + U[5]);
  }
  // memory-variable strain rates (k_curv_anelastic), PML-corrected from the
  // slabs' Q before this stage's Q update
  T e[6] = {0, 0, 0, 0, 0, 0}, tr = 0;
  if (RESP != RESP_EL && rhs) {
    e[0] = U[0]; e[1] = U[4]; e[2] = U[8];
    e[3] = U[3] + U[1]; e[4] = U[6] + U[2]; e[5] = U[7] + U[5];
    if (in_pml) {
      T dx, qx3, qx6, qx7, dy, qy4, qy6, qy8, dz, qz5, qz7, qz8;
      slab_strain<T, 0>(b, x, y, z, sx, 3, 6, 7, dx, qx3, qx6, qx7);
      slab_strain<T, 1>(b, x, y, z, sy, 4, 6, 8, dy, qy4, qy6, qy8);
      slab_strain<T, 2>(b, x, y, z, sz, 5, 7, 8, dz, qz5, qz7, qz8);
      e[0] = e[0] - dx * qx3;
      e[1] = e[1] - dy * qy4;
      e[2] = e[2] - dz * qz5;
      e[3] = e[3] - dx * qx6 - dy * qy6;
      e[4] = e[4] - dx * qx7 - dz * qz7;
      e[5] = e[5] - dy * qy8 - dz * qz8;
      tr = e[0] + e[1] + e[2];
    } else {
      tr = U[0] + U[4] + U[8];
    }
  }
  // PML damping and auxiliary fields, reference slab order z, y, x (before
  // the memory-variable sums here, so the derivative terms die before the
  // memory-variable stream: a rounding-level reordering of the rate sum)
  if (in_pml) {
    const GReg<T> G{U, S};
    if (rhs) {
      slab_pass<T, 2>(b, a, x, y, z, sz, true, integrate, sat, G, rhoJ_inv, lambda2mu, lam, mu, J, df);
      slab_pass<T, 1>(b, a, x, y, z, sy, true, integrate, sat, G, rhoJ_inv, lambda2mu, lam, mu, J, df);
      slab_pass<T, 0>(b, a, x, y, z, sx, true, integrate, sat, G, rhoJ_inv, lambda2mu, lam, mu, J, df);
    } else if (a.flags & (F_SCALE | F_UPDATE | F_SAT)) {
      slab_pass<T, 2>(b, a, x, y, z, sz, false, integrate, sat, G, (T)0, (T)0, (T)0, (T)0, (T)1, df);
      slab_pass<T, 1>(b, a, x, y, z, sy, false, integrate, sat, G, (T)0, (T)0, (T)0, (T)0, (T)1, df);
      slab_pass<T, 0>(b, a, x, y, z, sx, false, integrate, sat, G, (T)0, (T)0, (T)0, (T)0, (T)1, df);
    }
  }
  if (RESP != RESP_EL) {
    const T lm = rhs ? lam : b.M[p], mm = rhs ? mu : b.M[V + p];
    T s6[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    anelastic_lean<T, RESP>(b, a, x, y, z, p, lm, mm, e, tr, s6, rhs);
    if (rhs) {
#pragma unroll
      for (int c = 0; c < 6; ++c) df[3 + c] = df[3 + c] + s6[3 + c];
    }
  }
  if ((a.flags & F_SOURCE) && b.nsrc > 0 && x >= b.sbox[0] && x <= b.sbox[1] && y >= b.sbox[2] && y <= b.sbox[3] &&
      z >= b.sbox[4] && z <= b.sbox[5]) {
    const double t0 = a.time ? a.time->t : 0.0;
    const double tst = a.stage <= 1 ? t0 : t0 + c_rkC[a.stage - 1] * a.dt;
    add_sources<T, MESH_CURV>(b, tst, x, y, z, p, df);
  }
  if (sat && (x == 1 || x == b.nx || y == 1 || y == b.ny || z == 1 || z == b.nz)) {
    face_sat_add<T, 0>(b, x, y, z, df);
    face_sat_add<T, 1>(b, x, y, z, df);
    face_sat_add<T, 2>(b, x, y, z, df);
    face_sat_add<T, 3>(b, x, y, z, df);
    face_sat_add<T, 4>(b, x, y, z, df);
    face_sat_add<T, 5>(b, x, y, z, df);
  }
  if (a.flags & F_ISAT) {
    // interface SAT, src/RHS_Interior.f90:1813-1837: DF(face) -= tau0/hx * (F_x | G_x)
    const int side = x == 1 ? 0 : (x == b.nx ? 1 : -1);
    if (side >= 0 && b.isat[side]) {
      const T pen = b.tau0 / b.hq;
      const long long fp = (long long)(y - 1) + (long long)b.ny * (z - 1);
      const long long fn = (long long)b.ny * b.nz;
#pragma unroll
      for (int c = 0; c < 9; ++c) df[c] = df[c] - pen * b.isat[side][c * fn + fp];
    }
  }
#pragma unroll
  for (int c = 0; c < 9; ++c) DFp[c * V] = df[c];
  if (integrate) {
    const T Bdt = (T)a.Bdt;
    if (b.FC) {
#pragma unroll
      for (int c = 0; c < 9; ++c) {
        const T f0 = F[c * V + p];
        const T comp = b.FC[c * V + p];
        const T yv = Bdt * df[c] - comp;
        const T tv = f0 + yv;
        b.FC[c * V + p] = (tv - f0) - yv;
        Fn[c * V + p] = tv;
      }
    } else {
#pragma unroll
      for (int c = 0; c < 9; ++c) Fn[c * V + p] = F[c * V + p] + Bdt * df[c];
    }
  }
}

// Number of near-boundary (shell) points: everything outside the strict
// interior box, split into z-slabs, y-slabs of the middle planes and x-slabs
// of the middle rows.
template <typename T>
__host__ __device__ inline long long shell_count(const Blk<T> &b) {
  long long nx = b.nx, ny = b.ny;
  long long zlo = b.lo[2] - 1, zhi = b.nz - b.hi[2], nzm = b.hi[2] - b.lo[2] + 1;
  long long nym = b.hi[1] - b.lo[1] + 1;
  long long plane = nx * (b.lo[1] - 1) + nx * (b.ny - b.hi[1]) + nym * ((b.lo[0] - 1) + (b.nx - b.hi[0]));
  return nx * ny * (zlo + zhi) + (nzm > 0 ? nzm : 0) * plane;
}

template <typename T>
__device__ inline void shell_decode(const Blk<T> &b, int idx, int &x, int &y, int &z) {
  const int nx = b.nx, nxy = b.nx * b.ny;
  const int n_zlo = nxy * (b.lo[2] - 1), n_zhi = nxy * (b.nz - b.hi[2]);
  if (idx < n_zlo) {
    z = 1 + idx / nxy; int r = idx - (z - 1) * nxy; y = 1 + r / nx; x = 1 + r - (y - 1) * nx;
    return;
  }
  idx -= n_zlo;
  if (idx < n_zhi) {
    int zz = idx / nxy; z = b.hi[2] + 1 + zz; int r = idx - zz * nxy; y = 1 + r / nx; x = 1 + r - (y - 1) * nx;
    return;
  }
  idx -= n_zhi;
  const int ylo = nx * (b.lo[1] - 1), yhi = nx * (b.ny - b.hi[1]);
  const int wx = (b.lo[0] - 1) + (b.nx - b.hi[0]);
  const int nym = b.hi[1] - b.lo[1] + 1;
  const int plane = ylo + yhi + nym * wx;
  int zz = idx / plane;
  z = b.lo[2] + zz;
  int r = idx - zz * plane;
  if (r < ylo) { y = 1 + r / nx; x = 1 + r - (y - 1) * nx; return; }
  r -= ylo;
  if (r < yhi) { int yy = r / nx; y = b.hi[1] + 1 + yy; x = 1 + r - yy * nx; return; }
  r -= yhi;
  int yy = r / wx;
  y = b.lo[1] + yy;
  int c = r - yy * wx;
  x = c < (b.lo[0] - 1) ? 1 + c : b.hi[0] + 1 + (c - (b.lo[0] - 1));
}

template <typename T, int MESH, int RESP, bool SEP>
__global__ void __launch_bounds__(128, 3) k_shell(Blk<T> b, StageArgs a, int count) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= count) return;
  int x, y, z;
  shell_decode(b, idx, x, y, z);
  point_update<T, MESH, RESP, SEP, false, true>(b, a, x, y, z);
}


// ---------------------------------------------------------------------------
// Strict interior of a Cartesian block, src/JU_xJU_yJU_z6.f90:16426-16636,
// fused with scale, sources and the RK update; two warp groups per tile.
// 2.5-D: a block owns a 32 x TY column tile and marches up a z-chunk.  The
// nine outputs of a point are split: warps of group V (velocity rates)
// need z-derivatives of s_xz, s_yz, s_zz, warps of group S (stress rates) of
// v_x, v_y, v_z, so each thread's seven-plane z-queue is three fields and
// lives in registers.  Shared memory holds the double-buffered haloed x-y
// plane of eight fields, filled one plane ahead either by the tensor memory
// accelerator (TMA = true: one thread issues eight 4-D box loads of W x H
// points, x, y, z, component, completing on the buffer's mbarrier) or by
// 16-byte cp.async from every thread.
// ---------------------------------------------------------------------------
// smallest width >= w (a multiple of vec) whose h-row field plane is a whole
// number of 128-byte lines, so that every field's plane can be a TMA destination
constexpr int tma_plane_width(int w, int h, int esz, int vec) {
  while ((h * w * esz) % 128) w += vec;
  return w;
}

template <typename T, int TY, int NBUF = 2>
struct SplitSmem {
  static constexpr int VEC = 16 / (int)sizeof(T);
  static constexpr int H = TY + 6, NP = 32 * TY;
  static constexpr int W = tma_plane_width(((38 + VEC - 1 + VEC - 1) / VEC) * VEC, H, (int)sizeof(T), VEC);
  static constexpr int CH = W / VEC;
  static constexpr size_t plane_elems = (size_t)8 * H * W;
  // after the NBUF planes: the strain rates of the tile's points (6 x NP) and
  // the velocity group's memory-variable sums (3 x NP), anelastic blocks;
  // then the planes' mbarriers (TMA fills)
  static constexpr size_t bar_off = sizeof(T) * (NBUF * plane_elems + 9 * (size_t)NP);
  static constexpr size_t bytes = bar_off + NBUF * sizeof(uint64_t);
};

// polls of a TMA plane wait before the tile gives up (about a second)
constexpr int kTmaWaitLimit = 1 << 20;

// one 32 x TY column tile (tile indices bx, by, bz) of the strict interior;
// smraw is the planes' dynamic shared memory (1024-byte aligned for TMA);
// tm: the tensor map of the field buffer the stencil reads (TMA = true);
// NBUF plane buffers (cp.async: 2, filled one plane ahead; TMA: filled
// NBUF - 1 planes ahead)
template <typename T, int RESP, int TY, bool TMA = false, int NBUF = 2>
__device__ __forceinline__ void interior_split_tile(const Blk<T> &b, const StageArgs &a, int zchunk, int bx, int by,
                                                    int bz, unsigned char *smraw, const CUtensorMap *tm = nullptr) {
  static_assert(TMA || NBUF == 2, "cp.async fills use two plane buffers");
  using SM = SplitSmem<T, TY, NBUF>;
  constexpr int W = SM::W, H = SM::H, NP = SM::NP, VEC = SM::VEC, CH = SM::CH;
  constexpr int NT = 2 * NP;                                 // threads per block
  constexpr int NPOS = H * CH, PPT = (NPOS + NT - 1) / NT;
  T (*S)[8][H][W] = reinterpret_cast<T (*)[8][H][W]>(smraw);
  T *eb = reinterpret_cast<T *>(smraw) + NBUF * SM::plane_elems;   // strain rates, 6 x NP
  T *sb = eb + 6 * NP;                                           // memory-variable sums 3-5, 3 x NP
  uint64_t *bars = reinterpret_cast<uint64_t *>(smraw + SM::bar_off);
  const int tid = threadIdx.x;
  const bool gS = tid >= NP;                                 // stress-rate group
  const int lt = gS ? tid - NP : tid;
  const int tx = lt & 31, ty = lt >> 5;
  const int x0 = b.lo[0] + bx * 32;
  const int y0 = b.lo[1] + by * TY;
  const int zs = b.lo[2] + bz * zchunk;
  if (zs > b.hi[2]) return;
  const int ze = min(zs + zchunk - 1, b.hi[2]);
  const int x = x0 + tx, y = y0 + ty;
  const bool active = x <= b.hi[0] && y <= b.hi[1];
  const long long V = b.vol;
  const T *F = a.cur ? b.F1 : b.F0;
  T *Fn = a.cur ? b.F0 : b.F1;
  const double t0 = a.time ? a.time->t : 0.0;
  const double tst = a.stage <= 1 ? t0 : t0 + c_rkC[a.stage - 1] * a.dt;
  const long long pc = pidx(b, min(x, b.nx), min(y, b.ny), zs);
  const long long row0 = pidx(b, x0 - 3, y0 - 3, zs);
  const int sh = (int)(row0 % VEC);
  const long long base0 = row0 - sh;
  const long long rowstart0 = base0 - ((base0 % b.sz) % b.sy);
  int soff[PPT];
  long long goff[PPT];
  bool gok[PPT];
#pragma unroll
  for (int k = 0; k < PPT; ++k) {
    int pos = tid + k * NT;
    int yy = pos / CH, ch = pos - yy * CH;
    soff[k] = yy * W + ch * VEC;
    goff[k] = (long long)yy * b.sy + (long long)ch * VEC;
    long long inrow = base0 - rowstart0 + (long long)ch * VEC;
    gok[k] = pos < NPOS && (y0 - 3 + yy) <= b.ny + 3 && inrow + VEC <= b.sy;
  }
  bool stalled = false;
  if constexpr (TMA) {
    if (tid == 0) {
#pragma unroll
      for (int k = 0; k < NBUF; ++k) mbar_init(&bars[k], 1);
      mbar_init_fence();
    }
    __syncthreads();
  }
  auto fill = [&](int zz, int buf) {
    const long long plane0 = base0 + (long long)(zz - zs) * b.sz;
    T *dst = &S[buf][0][0][0];
    if constexpr (TMA) {
      // box origin (x, y, z, component) of the plane in the padded array;
      // base0 is 16-byte aligned and the row / plane pitches are multiples of
      // 128 bytes, so x is too; a violated rule issues no copy and the
      // bounded wait records the stall
      if (tid == 0) {
        const long long rem = plane0 % b.sz;
        const int cx = (int)(rem % b.sy), cy = (int)(rem / b.sy), cz = (int)(plane0 / b.sz);
        if ((cx % VEC) == 0 && (smem_u32(dst) & 127u) == 0 && !a.nofill) {
          mbar_expect_tx(&bars[buf], (unsigned)(8 * H * W * sizeof(T)));
#pragma unroll
          for (int f = 0; f < 8; ++f) tma_load_4d(dst + f * H * W, tm, cx, cy, cz, c_smf[f], &bars[buf]);
        }
      }
    } else {
#pragma unroll
      for (int f = 0; f < 8; ++f) {
        const T *srcf = F + c_smf[f] * V + plane0;
#pragma unroll
        for (int k = 0; k < PPT; ++k)
          if (tid + k * NT < NPOS) cp_async<16>(dst + f * H * W + soff[k], gok[k] ? srcf + goff[k] : F, gok[k]);
      }
    }
  };
  // z-queue fields: group V -> s_zz, s_xz, s_yz (F 5, 7, 8); group S -> v_x, v_y, v_z (F 0, 1, 2)
  const int q0 = gS ? 0 : 5, q1 = gS ? 1 : 7, q2 = gS ? 2 : 8;
  T q[3][7];
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const long long pz = pc + (long long)(k - 3) * b.sz;
    q[0][k] = ld(F + q0 * V + pz);
    q[1][k] = ld(F + q1 * V + pz);
    q[2][k] = ld(F + q2 * V + pz);
  }
  q[0][6] = ld(F + q0 * V + pc + 3 * b.sz);
  q[1][6] = ld(F + q1 * V + pc + 3 * b.sz);
  q[2][6] = ld(F + q2 * V + pc + 3 * b.sz);
  fill(zs, 0);
  if constexpr (TMA) {
#pragma unroll
    for (int k = 1; k < NBUF - 1; ++k)
      if (zs + k <= ze) fill(zs + k, k);
  } else {
    cp_async_commit();
  }
  // this group's rates and material, one step ahead
  const int nd = gS ? 6 : 3, d0 = gS ? 3 : 0;
  // FP32 (compensated) path: the update's global operands -- the compensation
  // and sigma_zz of group S, which the staged plane does not hold -- also one
  // plane ahead (FP64 keeps its registers for the stencil)
  constexpr bool PRE = sizeof(T) == 4;
  // the rates of the next plane read one plane ahead, except in FP64 blocks
  // with 8 mechanisms (registers for the memory-variable stream)
  constexpr bool DFPRE = PRE || RESP == RESP_EL || RESP == RESP_Q4;
  constexpr int NPRE = PRE ? 6 : 1;
  const bool upd = (a.flags & F_UPDATE) != 0, kahan = PRE && upd && b.FC != nullptr;
  T dfo[6], m0 = 0, m1 = 0, fco[NPRE], szo = 0;
  if (active) {
#pragma unroll
    for (int c = 0; c < 6; ++c) dfo[c] = c < nd ? b.DF[(d0 + c) * V + pc] : (T)0;
    if (gS) { m0 = b.M[pc]; m1 = b.M[V + pc]; } else { m0 = b.M[2 * V + pc]; }
    if constexpr (PRE) {
#pragma unroll
      for (int c = 0; c < NPRE; ++c) fco[c] = (kahan && c < nd) ? b.FC[(d0 + c) * V + pc] : (T)0;
      if (upd && gS) szo = ld(F + 5 * V + pc);
    }
  }
  const T mx = active ? ld(b.mq + x) : (T)0, my = active ? ld(b.mr + y) : (T)0;

  for (int z = zs; z <= ze; ++z) {
    const int i = z - zs;
    const int buf = TMA ? i % NBUF : (i & 1);
    const long long p = pc + (long long)i * b.sz;
    if constexpr (TMA) {
      // the plane of this iteration: buffer buf's (i / NBUF)-th fill (after a
      // wait that gave up, the tile no longer waits)
      if (!stalled && !mbar_wait_bounded(&bars[buf], (unsigned)((i / NBUF) & 1), kTmaWaitLimit)) stalled = true;
    } else {
      cp_async_wait_all();
    }
    __syncthreads();
    if constexpr (TMA) {
      // the buffer of iteration i - 1, which every thread has left
      if (z + NBUF - 1 <= ze) fill(z + NBUF - 1, (i + NBUF - 1) % NBUF);
    } else {
      if (z + 1 <= ze) fill(z + 1, buf ^ 1);
      cp_async_commit();
    }
    T qn0 = 0, qn1 = 0, qn2 = 0, dfn[6], mn0 = 0, mn1 = 0, fcn[NPRE], szn = 0;
    if (z + 1 <= ze) {
      const long long pn = p + 4 * b.sz;
      qn0 = ld(F + q0 * V + pn); qn1 = ld(F + q1 * V + pn); qn2 = ld(F + q2 * V + pn);
      if (active) {
#pragma unroll
        for (int c = 0; c < 6; ++c) dfn[c] = (DFPRE && c < nd) ? b.DF[(d0 + c) * V + p + b.sz] : (T)0;
        if (gS) { mn0 = b.M[p + b.sz]; mn1 = b.M[V + p + b.sz]; } else { mn0 = b.M[2 * V + p + b.sz]; }
        if constexpr (PRE) {
#pragma unroll
          for (int c = 0; c < NPRE; ++c) fcn[c] = (kahan && c < nd) ? b.FC[(d0 + c) * V + p + b.sz] : (T)0;
          if (upd && gS) szn = ld(F + 5 * V + p + b.sz);
        }
        if (RESP != RESP_EL && (PRE || b.nmech <= 4)) {
          // the next plane's memory variables of this group's stress
          // components, read late by anelastic_lean (FP64: Q4 only; measured
          // 10 % faster on Q4 shots, 21 % slower on the fQ8 planar blocks)
          const int nmv = 3 * b.nmech, cm0 = gS ? 0 : nmv;
          for (int c = cm0; c < cm0 + nmv; ++c) {
            prefetch_l2(b.eta + (long long)c * V + p + b.sz);
            prefetch_l2(b.deta + (long long)c * V + p + b.sz);
          }
        }
      }
    }
    const T(*P)[H][W] = S[buf];
    const int c0 = tx + sh + 3, r0 = ty + 3;
    if (!DFPRE && active) {
#pragma unroll
      for (int c = 0; c < 6; ++c) dfo[c] = c < nd ? b.DF[(d0 + c) * V + p] : (T)0;
    }
    T df[9];                                                 // group S: stress rates 3..8
    if (active) {
      const T mz = ld(b.ms + z);
#define DX(f) (((T)0 + (mx * b.cx[0]) * (P[f][r0][c0 + 1] - P[f][r0][c0 - 1])) + \
               (mx * b.cx[1]) * (P[f][r0][c0 + 2] - P[f][r0][c0 - 2])) + \
              (mx * b.cx[2]) * (P[f][r0][c0 + 3] - P[f][r0][c0 - 3])
#define DY(f) (((T)0 + (my * b.cy[0]) * (P[f][r0 + 1][c0] - P[f][r0 - 1][c0])) + \
               (my * b.cy[1]) * (P[f][r0 + 2][c0] - P[f][r0 - 2][c0])) + \
              (my * b.cy[2]) * (P[f][r0 + 3][c0] - P[f][r0 - 3][c0])
#define DZ(k) (((T)0 + (mz * b.cz[0]) * (q[k][4] - q[k][2])) + (mz * b.cz[1]) * (q[k][5] - q[k][1])) + \
              (mz * b.cz[2]) * (q[k][6] - q[k][0])
      const T Bdt = (T)a.Bdt;
      const bool sc = (a.flags & F_SCALE) != 0;
      if (!gS) {
        // velocity rates: a1 * (d sxx/dx + d sxy/dy + d sxz/dz), ...   (queue: 0 szz, 1 sxz, 2 syz)
        const T a1 = (T)1 / m0;
        T df0 = sc ? (T)a.A * dfo[0] : dfo[0];
        T df1 = sc ? (T)a.A * dfo[1] : dfo[1];
        T df2 = sc ? (T)a.A * dfo[2] : dfo[2];
        df0 = df0 + a1 * (DX(3) + DY(5) + DZ(1));
        df1 = df1 + a1 * (DX(5) + DY(4) + DZ(2));
        df2 = df2 + a1 * (DX(6) + DY(7) + DZ(0));
        b.DF[0 * V + p] = df0;
        b.DF[1 * V + p] = df1;
        b.DF[2 * V + p] = df2;
        if (a.flags & F_UPDATE) {
          const T f0 = P[0][r0][c0], f1 = P[1][r0][c0], f2 = P[2][r0][c0];
          if (b.FC) {
            const T dv[3] = {df0, df1, df2}, fv[3] = {f0, f1, f2};
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              T comp = PRE ? fco[c % NPRE] : b.FC[c * V + p];
              T yv = Bdt * dv[c] - comp;
              T tv = fv[c] + yv;
              b.FC[c * V + p] = (tv - fv[c]) - yv;
              Fn[c * V + p] = tv;
            }
          } else {
            Fn[0 * V + p] = f0 + Bdt * df0;
            Fn[1 * V + p] = f1 + Bdt * df1;
            Fn[2 * V + p] = f2 + Bdt * df2;
          }
        }
      } else {
        // stress rates from velocity gradients (queue: 0 vx, 1 vy, 2 vz)
        const T lam = m0, mu = m1;
        const T a2 = (T)2 * mu + lam, a3 = lam, a4 = mu;
        const T vxx = DX(0), vyx = DX(1), vzx = DX(2);
        const T vxy = DY(0), vyy = DY(1), vzy = DY(2);
        const T vxz = DZ(0), vyz = DZ(1), vzz = DZ(2);
#pragma unroll
        for (int c = 0; c < 6; ++c) df[3 + c] = sc ? (T)a.A * dfo[c] : dfo[c];
        df[3] = df[3] + a2 * vxx + a3 * (vyy + vzz);
        df[4] = df[4] + a2 * vyy + a3 * (vxx + vzz);
        df[5] = df[5] + a2 * vzz + a3 * (vxx + vyy);
        df[6] = df[6] + a4 * (vxy + vyx);
        df[7] = df[7] + a4 * (vxz + vzx);
        df[8] = df[8] + a4 * (vyz + vzy);
        if (RESP != RESP_EL) {
          // the strain rates to shared memory: the memory variables of stress
          // components 0-2 are this group's, 3-5 the velocity group's
          eb[0 * NP + lt] = vxx; eb[1 * NP + lt] = vyy; eb[2 * NP + lt] = vzz;
          eb[3 * NP + lt] = vxy + vyx; eb[4 * NP + lt] = vxz + vzx; eb[5 * NP + lt] = vyz + vzy;
        }
      }
#undef DX
#undef DY
#undef DZ
    }
    if constexpr (RESP != RESP_EL) {
      // lean memory-variable update (per-point factors, 1/tau multiplied),
      // stress components split between the two groups
      __syncthreads();
      if (active) {
        T e[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) e[c] = eb[c * NP + lt];
        const T tr = e[0] + e[1] + e[2];
        if (gS) {
          anelastic_lean<T, RESP, 0, 3>(b, a, x, y, z, p, m0, m1, e, tr, df, true);
        } else {
          T s9[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
          anelastic_lean<T, RESP, 3, 6>(b, a, x, y, z, p, b.M[p], b.M[V + p], e, tr, s9, true);
          sb[0 * NP + lt] = s9[6]; sb[1 * NP + lt] = s9[7]; sb[2 * NP + lt] = s9[8];
        }
      }
      __syncthreads();
      if (active && gS) {
        df[6] = df[6] + sb[0 * NP + lt];
        df[7] = df[7] + sb[1 * NP + lt];
        df[8] = df[8] + sb[2 * NP + lt];
      }
    }
    if (active && gS) {
      {
        const T Bdt = (T)a.Bdt;
        if ((a.flags & F_SOURCE) && b.nsrc > 0 && x >= b.sbox[0] && x <= b.sbox[1] && y >= b.sbox[2] &&
            y <= b.sbox[3] && z >= b.sbox[4] && z <= b.sbox[5]) {
          df[0] = df[1] = df[2] = (T)0;
          add_sources<T, MESH_CART>(b, tst, x, y, z, p, df);
        }
#pragma unroll
        for (int c = 3; c < 9; ++c) b.DF[c * V + p] = df[c];
        if (a.flags & F_UPDATE) {
          T fc[9];
          fc[3] = P[3][r0][c0]; fc[4] = P[4][r0][c0];
          fc[5] = PRE ? szo : ld(F + 5 * V + p);
          fc[6] = P[5][r0][c0]; fc[7] = P[6][r0][c0]; fc[8] = P[7][r0][c0];
          if (b.FC) {
#pragma unroll
            for (int c = 3; c < 9; ++c) {
              T comp = PRE ? fco[(c - 3) % NPRE] : b.FC[c * V + p];
              T yv = Bdt * df[c] - comp;
              T tv = fc[c] + yv;
              b.FC[c * V + p] = (tv - fc[c]) - yv;
              Fn[c * V + p] = tv;
            }
          } else {
#pragma unroll
            for (int c = 3; c < 9; ++c) Fn[c * V + p] = fc[c] + Bdt * df[c];
          }
        }
      }
    }
    // advance the queue and the prefetched values
#pragma unroll
    for (int k = 0; k < 6; ++k) { q[0][k] = q[0][k + 1]; q[1][k] = q[1][k + 1]; q[2][k] = q[2][k + 1]; }
    q[0][6] = qn0; q[1][6] = qn1; q[2][6] = qn2;
#pragma unroll
    for (int c = 0; c < 6; ++c) dfo[c] = dfn[c];
    if constexpr (PRE) {
#pragma unroll
      for (int c = 0; c < NPRE; ++c) fco[c] = fcn[c];
      szo = szn;
    }
    m0 = mn0; m1 = mn1;
  }
  if constexpr (!TMA) cp_async_wait_all();
  if (stalled && a.time) atomicOr(const_cast<int *>(&a.time->stall), 1);
}

template <typename T, int RESP, int TY, bool TMA, int NBUF>
__global__ void __launch_bounds__(64 * TY, (TY == 4 ? 2 : 1))
    k_interior_split(Blk<T> b, StageArgs a, int zchunk, const __grid_constant__ CUtensorMap tm) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  interior_split_tile<T, RESP, TY, TMA, NBUF>(b, a, zchunk, blockIdx.x, blockIdx.y, blockIdx.z, smraw, &tm);
}

// F <- F + dt*DF over every interior point (update_fields, split path): in place
template <typename T>
__global__ void k_update_inplace(Blk<T> b, int cur, double dt) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int y = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int z = blockIdx.z * blockDim.z + threadIdx.z + 1;
  if (x > b.nx || y > b.ny || z > b.nz) return;
  const long long p = pidx(b, x, y, z);
  T *F = cur ? b.F1 : b.F0;
  const T d = (T)dt;
  for (int c = 0; c < 9; ++c) F[c * b.vol + p] = F[c * b.vol + p] + d * b.DF[c * b.vol + p];
}

// rk_vector_openacc.f90:22-37 / :58-75 equivalents on flat device arrays
static __global__ void k_scale_array(double *r, long long n, double A) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long s = (long long)gridDim.x * blockDim.x;
  for (; i < n; i += s) r[i] = A * r[i];
}
static __global__ void k_axpy_array(double *x, const double *r, long long n, double dt) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long s = (long long)gridDim.x * blockDim.x;
  for (; i < n; i += s) x[i] = x[i] + dt * r[i];
}
template <typename T>
__global__ void k_scale_T(T *r, long long n, double A) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long s = (long long)gridDim.x * blockDim.x;
  for (; i < n; i += s) r[i] = (T)A * r[i];
}
template <typename T>
__global__ void k_axpy_T(T *x, const T *r, long long n, double dt) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long s = (long long)gridDim.x * blockDim.x;
  for (; i < n; i += s) x[i] = x[i] + (T)dt * r[i];
}

// Receiver gather at the start of step n (stage 1, before the update) and
// time advance at the end of a step.
template <typename T>
__device__ __forceinline__ void sample_block(const Blk<T> &b, int cur, DevTime *tm, int w_stride, int increment) {
  const T *F = cur ? b.F1 : b.F0;
  int n = tm->n;
  if (w_stride <= 0 || ((n - 1) % w_stride) != 0) return;
  int s = tm->nsamp;
  if (s < b.max_samples) {
    for (int r = threadIdx.x; r < b.nrec; r += blockDim.x) {
      double *o = b.seis + ((long long)s * b.nrec + r) * 4;
      int i = b.ridx[3 * r], j = b.ridx[3 * r + 1], k = b.ridx[3 * r + 2];
      o[0] = tm->t;
      if (i > 0 && j > 0 && k > 0) {
        long long p = pidx(b, i, j, k);
        o[1] = (double)F[p];
        o[2] = (double)F[b.vol + p];
        o[3] = (double)F[2 * b.vol + p];
        // the reference stops a run whose station values are not finite
        // (src/seismogram.f90:516-524, RUN-STATION-001): flag the first such step
        if (!(fabs(o[1]) <= 1.7976931348623157e308 && fabs(o[2]) <= 1.7976931348623157e308 &&
              fabs(o[3]) <= 1.7976931348623157e308))
          atomicCAS(&tm->bad, 0, n);
      } else {
        o[1] = o[2] = o[3] = 0.0;
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0 && increment) tm->nsamp = s + 1;
}

template <typename T>
__global__ void k_sample(Blk<T> b, int cur, DevTime *tm, int w_stride, int increment) {
  sample_block<T>(b, cur, tm, w_stride, increment);
}

static __global__ void k_advance(DevTime *tm, double dt) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    tm->t = tm->t + c_rkC[5] * dt;
    tm->n = tm->n + 1;
  }
}

// max |v| reduction (final-state diagnostics) with a non-finite flag
template <typename T>
__global__ void k_maxabs(const T *a, long long n, double *partial, int *nonfinite) {
  __shared__ double sm[256];
  double m = 0.0;
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long s = (long long)gridDim.x * blockDim.x;
  int bad = 0;
  for (; i < n; i += s) {
    double v = fabs((double)a[i]);
    if (!(v <= 1.7976931348623157e308)) bad = 1;
    else if (v > m) m = v;
  }
  sm[threadIdx.x] = m;
  if (bad) atomicExch(nonfinite, 1);
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + k]);
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sm[0];
}

}  // namespace wql3d
