// Block-interface coupling on the q-direction interface between two blocks.
//
// One thread per interface point (y, z) does, for both sides of the fault,
// what the reference does in Impose_Interface_Condition / Couple_Interface_x /
// Interface_RHS (src/RHS_Interior.f90:1771-1843, src/CouplingForcing.f90:9-463,
// src/Interface_Condition.f90:12-916):
//   tractions from the face stresses, rotation to the (n, m, l) basis of the
//   calling block's face, the interface law (locked, linear friction or
//   linear slip-weakening friction with its prestress and strength), the
//   stage-1 fault outputs, rotation back and the characteristic SAT vector
//   of the calling side.
// Side 1 (the reference's ib = 2) is block 1's q-max face and side 2 (ib = 1)
// block 2's q-min face; both read the same two face traces and each uses its
// own face basis, metric and coordinates, as the reference's two calls do.
// The SAT vectors go to sat_m / sat_p, which the stage kernels subtract at the
// face points (DF -= tau0/hq * sat) after the physical-boundary SATs.
//
// Slip S (3 components + cumulative |V|) and the state W live here in FP64
// for both field precisions: S = S + B dt DS after DS = A DS + (Q - P).
// The friction law reads S before this stage's update, like Interface_RHS
// reads I%S before update_fields.
#pragma once

#include <cmath>
#include <vector>

#include "wql3d.h"
#include "wql3d_device.cuh"

namespace wql3d {

struct IfaceDev {
  int ny = 0, nz = 0;
  int coupling = WQL3D_IFACE_LOCKED;
  int serial = 0;          // 1: both sides accumulate DS (one-process two-block reading)
  double fd = 0.525, Dc = 0.4;
  double *S = nullptr, *DS = nullptr;     // 4 x n
  double *W = nullptr, *DW = nullptr;     // n
  double *Svel = nullptr;                 // 3 x n (stage 1)
  double *Uhat = nullptr, *Vhat = nullptr;// 6 x n (stage 1)
  double *trup = nullptr;                 // n
  double *t0[2] = {nullptr, nullptr};     // per side: 3 x n initial tractions n, m, l
  double *fs[2] = {nullptr, nullptr};     // per side: n static friction
  void *sat_m = nullptr;   // SAT vector added at block 1's q-max face (F_x)
  void *sat_p = nullptr;   // SAT vector added at block 2's q-min face (G_x)
  // remote interface side: this domain holds one block, side `remote` (1: its
  // q-max face, 2: its q-min face); the other side's face trace and material
  // arrive in recv / oppM
  int remote = 0;
  void *send = nullptr;    // this block's face trace, 9 x n (field precision)
  void *recv = nullptr;    // the other side's face trace, 9 x n
  void *oppM = nullptr;    // the other side's lambda, mu, rho at the face, 3 x n
  // rate-and-state (TPV101 / TPV102): per side the direct-effect map a and the
  // nucleation amplitude 25 F(r) of the time-ramped prestress
  double *ra[2] = {nullptr, nullptr};
  double *nuc[2] = {nullptr, nullptr};
};

// TPV101 / TPV102 rate-and-state parameters, src/Interface_Condition.f90:386-401
constexpr double kRsL0 = 0.02, kRsF0 = 0.6, kRsB = 0.012, kRsV0 = 1.0e-6;

// smooth_boxcar, src/Interface_Condition.f90:2460-2476
inline double host_smooth_boxcar(double x, double w, double wr) {
  if (-w <= x && x <= w) return 1.0;
  if (std::fabs(x) > w && std::fabs(x) < w + wr)
    return 0.5 * (1.0 + std::tanh(wr / (std::fabs(x) - w - wr) + wr / (std::fabs(x) - w)));
  return 0.0;
}

// per-point direct-effect parameter a and nucleation amplitude 25 F(r)
// (src/Interface_Condition.f90:386-401, 2340-2352)
inline void rs_point(const double x[3], double *a, double *nuc) {
  *a = 0.008 + 0.008 * (1.0 - host_smooth_boxcar(x[1], 15.0, 3.0) * host_smooth_boxcar(x[2], 15.0, 3.0));
  const double r = std::sqrt((x[1] - 7.5) * (x[1] - 7.5) + x[2] * x[2]);
  double F = 0.0;
  if (r < 3.0) F = std::exp(r * r / (r * r - 9.0));
  *nuc = 25.0 * F;
}

inline bool rs_problem(int p) { return p == WQL3D_FAULT_TPV101 || p == WQL3D_FAULT_TPV102; }

// boxcar of unit amplitude on (-w, w), 1/2 within 100 eps of the edges
// (src/Interface_Condition.f90:2438-2457)
inline double host_boxcar(double x, double w) {
  const double tol = 100.0 * 2.220446049250313e-16;
  if (-w + tol < x && x < w - tol) return 1.0;
  if (std::fabs(-w - x) <= tol || std::fabs(x - w) <= tol) return 0.5;
  return 0.0;
}

// TPV5 prestress and static friction at one fault point
// (src/Interface_Condition.f90:1822-1830 and 1283-1294)
inline void tpv5_point(const double x[3], double *T0n, double *T0m, double *T0l, double *fs) {
  double tl = 70.0;
  tl = tl + 8.0 * host_boxcar(x[1] - 7.5, 1.5) * host_boxcar(x[2] + 7.5, 1.5);
  tl = tl + 11.6 * host_boxcar(x[1] - 7.5, 1.5) * host_boxcar(x[2], 1.5);
  tl = tl - 8.0 * host_boxcar(x[1] - 7.5, 1.5) * host_boxcar(x[2] - 7.5, 1.5);
  *T0n = -120.0;
  *T0m = 0.0;
  *T0l = tl;
  *fs = 0.677 + 1.0e10 * (1.0 - host_boxcar(x[1], 15.0) * host_boxcar(x[2], 15.0));
}

// TPV28 background stress (src/initial_stress_condition.f90:78-84), unless
// the description gives one
inline const double *tpv28_stress(const wql3d_domain_desc &desc) {
  static const double s0[6] = {-60.0, 0.0, 60.0, 0.0, 29.38, 0.0};
  for (int c = 0; c < 6; ++c)
    if (desc.fault_stress[c] != 0.0) return desc.fault_stress;
  return s0;
}

// TPV28 prestress and static friction at one fault point
// (src/Interface_Condition.f90:2049-2076 and 1459-1474): the stress tensor
// as tractions on n, rotated onto (n, m, l), plus the nucleation shear on T0_l
inline void tpv28_point(const double s0[6], const double x[3], const double n[3], const double m[3],
                        const double l[3], double *T0n, double *T0m, double *T0l, double *fs) {
  const double sxx = s0[0], syy = s0[1], szz = s0[2], sxy = s0[3], sxz = s0[4], syz = s0[5];
  const double Tx = n[0] * sxx + n[1] * sxy + n[2] * sxz;
  const double Ty = n[0] * sxy + n[1] * syy + n[2] * syz;
  const double Tz = n[0] * sxz + n[1] * syz + n[2] * szz;
  *T0n = n[0] * Tx + n[1] * Ty + n[2] * Tz;
  *T0m = m[0] * Tx + m[1] * Ty + m[2] * Tz;
  *T0l = l[0] * Tx + l[1] * Ty + l[2] * Tz;
  const double r = std::sqrt((x[1] - 7.5) * (x[1] - 7.5) + x[2] * x[2]);
  double nuke = 0.0;
  if (r <= 1.4) nuke = 11.60;
  else if (r >= 1.4 && r <= 2.0) nuke = 5.8 * (1.0 + std::cos(3.141592653589793 * (r - 1.4) / 0.6));
  *T0l = *T0l + nuke;
  *fs = 0.677 + 1.0e10 * (1.0 - host_boxcar(x[1], 15.0) * host_boxcar(x[2], 18.0));
}

// fault_problem range check shared by the interface setups
inline bool fault_problem_ok(const wql3d_domain_desc &desc) {
  if (desc.coupling < WQL3D_IFACE_LOCKED || desc.coupling > WQL3D_IFACE_RATE_STATE) return false;
  if (desc.fault_problem < WQL3D_FAULT_MAPS || desc.fault_problem > WQL3D_FAULT_TPV28) return false;
  return (desc.coupling == WQL3D_IFACE_RATE_STATE) == rs_problem(desc.fault_problem);
}

// slip-weakening fd and Dc: the problem's own (TPV5 0.525 / 0.4, TPV28
// 0.373 / 0.4; src/Interface_Condition.f90:1283-1299, 1459-1474) or the
// description's
inline void fault_weakening(const wql3d_domain_desc &desc, double *fd, double *Dc) {
  *fd = desc.fd;
  *Dc = desc.Dc;
  if (desc.fault_problem == WQL3D_FAULT_TPV5) { *fd = 0.525; *Dc = 0.4; }
  if (desc.fault_problem == WQL3D_FAULT_TPV28) { *fd = 0.373; *Dc = 0.4; }
}

// Per-point prestress / strength maps of one block's interface face (face 1:
// its q-max face at q = xend = nq, face 0: its q-min face), and the
// rate-and-state a and nucleation maps.  The TPV28 prestress is projected on
// the block's own face basis, as each side's Interface_RHS call does.
template <typename T>
int fault_maps(const wql3d_domain_desc &desc, const Blk<T> &b, int face, const std::vector<double> &coords, int xend,
               std::vector<double> &t0, std::vector<double> &f, std::vector<double> &ra, std::vector<double> &nuc,
               cudaStream_t s) {
  const int ny = b.ny, nz = b.nz;
  const long long n = (long long)ny * nz;
  t0.assign((size_t)(3 * n), 0.0);
  f.assign((size_t)n, desc.fs);
  ra.assign((size_t)n, 0.0);
  nuc.assign((size_t)n, 0.0);
  std::vector<T> B;
  if (desc.fault_problem == WQL3D_FAULT_TPV28) {
    B.resize((size_t)(9 * n));
    if (cudaMemcpyAsync(B.data(), b.nrm[face], sizeof(T) * 9 * n, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return WQL3D_ECUDA;
  }
  const double *s0 = tpv28_stress(desc);
  const long long nb = (long long)b.nx * ny * nz;
  for (int z = 1; z <= nz; ++z)
    for (int y = 1; y <= ny; ++y) {
      const long long k = (long long)(y - 1) + (long long)ny * (z - 1);
      const long long q = (long long)(xend - 1) + (long long)b.nx * ((y - 1) + (long long)ny * (z - 1));
      const double x[3] = {coords[(size_t)q], coords[(size_t)(nb + q)], coords[(size_t)(2 * nb + q)]};
      if (rs_problem(desc.fault_problem)) {
        rs_point(x, &ra[(size_t)k], &nuc[(size_t)k]);
      } else if (desc.fault_problem == WQL3D_FAULT_TPV5) {
        tpv5_point(x, &t0[(size_t)k], &t0[(size_t)(n + k)], &t0[(size_t)(2 * n + k)], &f[(size_t)k]);
      } else if (desc.fault_problem == WQL3D_FAULT_TPV28) {
        double l[3], m[3], nv[3];
        for (int c = 0; c < 3; ++c) {
          l[c] = (double)B[(size_t)((0 + c) * n + k)];
          m[c] = (double)B[(size_t)((3 + c) * n + k)];
          nv[c] = (double)B[(size_t)((6 + c) * n + k)];
        }
        tpv28_point(s0, x, nv, m, l, &t0[(size_t)k], &t0[(size_t)(n + k)], &t0[(size_t)(2 * n + k)], &f[(size_t)k]);
      } else {
        if (desc.iface_tau0)
          for (int c = 0; c < 3; ++c) t0[(size_t)(c * n + k)] = desc.iface_tau0[c * n + k];
        if (desc.iface_fs) f[(size_t)k] = desc.iface_fs[k];
      }
    }
  return WQL3D_OK;
}

// init_vel_state's state for TPV101 / TPV102 (src/Interface_Condition.f90:2722-2786):
// W from the t = 0 traction on one block's interface face (basis of face
// `face`, coordinates at q = xend): theta = L0/V0 exp((a log(2 sinh(T0_l/(a
// sigma_n))) - f0 - a log(Vin/V0))/b), W = f0 + b log(V0/L0 theta).  V0 is an
// unsuffixed literal there: single precision unless reals are promoted (lit).
template <typename T>
int rs_init_state(IfaceDev &I, const Blk<T> &b, int face, const std::vector<double> &coords, int xend, cudaStream_t s) {
  const int ny = I.ny, nz = I.nz;
  const long long n = (long long)ny * nz;
  std::vector<T> B((size_t)(9 * n));
  if (cudaMemcpyAsync(B.data(), b.nrm[face], sizeof(T) * 9 * n, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return WQL3D_ECUDA;
  const double Vin = 1.0e-12, V0 = b.lit ? (double)1.0e-6f : 1.0e-6;
  const double sxx = -120.0, syy = 0.0, szz = -120.0, sxy = 0.0, sxz = 75.0, syz = 0.0;
  const long long nb = (long long)b.nx * ny * nz;
  std::vector<double> W((size_t)n);
  for (int z = 1; z <= nz; ++z)
    for (int y = 1; y <= ny; ++y) {
      const long long k = (long long)(y - 1) + (long long)ny * (z - 1);
      const long long q = (long long)(xend - 1) + (long long)b.nx * ((y - 1) + (long long)ny * (z - 1));
      const double x[3] = {coords[(size_t)q], coords[(size_t)(nb + q)], coords[(size_t)(2 * nb + q)]};
      double l[3], m[3], nv[3];
      for (int c = 0; c < 3; ++c) {
        l[c] = (double)B[(size_t)((0 + c) * n + k)];
        m[c] = (double)B[(size_t)((3 + c) * n + k)];
        nv[c] = (double)B[(size_t)((6 + c) * n + k)];
      }
      const double Tx = nv[0] * sxx + nv[1] * sxy + nv[2] * sxz;
      const double Ty = nv[0] * sxy + nv[1] * syy + nv[2] * syz;
      const double Tz = nv[0] * sxz + nv[1] * syz + nv[2] * szz;
      const double T0n = nv[0] * Tx + nv[1] * Ty + nv[2] * Tz;
      const double T0l = l[0] * Tx + l[1] * Ty + l[2] * Tz;
      (void)m;
      double a, nuc;
      rs_point(x, &a, &nuc);
      const double sigma_n = -T0n;
      const double theta = kRsL0 / V0 *
                           std::exp(((a * std::log(2.0 * std::sinh(T0l / (a * sigma_n)))) - kRsF0 - a * std::log(Vin / V0)) / kRsB);
      W[(size_t)k] = kRsF0 + kRsB * std::log(V0 / kRsL0 * theta);
    }
  if (cudaMemcpyAsync(I.W, W.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return WQL3D_ECUDA;
  return WQL3D_OK;
}

// Allocate the interface state and build the per-side prestress / strength
// maps.  coords0 / coords1: host coordinates of the two blocks (3 x nq*nr*ns,
// x fastest); nq0 is block 1's q extent.
template <typename T, typename AllocT>
int setup_iface(IfaceDev &I, const wql3d_domain_desc &desc, const Blk<T> &b0, const Blk<T> &b1,
                const std::vector<double> &coords0, const std::vector<double> &coords1, AllocT &mem,
                cudaStream_t s) {
  if (b0.ny != b1.ny || b0.nz != b1.nz) return WQL3D_EINVAL;
  if (!fault_problem_ok(desc)) return WQL3D_EINVAL;
  const int ny = b0.ny, nz = b0.nz;
  const long long n = (long long)ny * nz;
  I.ny = ny;
  I.nz = nz;
  I.coupling = desc.coupling;
  I.serial = desc.serial_shared ? 1 : 0;
  fault_weakening(desc, &I.fd, &I.Dc);
  if (mem.get(&I.S, 4 * n) || mem.get(&I.DS, 4 * n) || mem.get(&I.W, n) || mem.get(&I.DW, n) ||
      mem.get(&I.Svel, 3 * n) || mem.get(&I.Uhat, 6 * n) || mem.get(&I.Vhat, 6 * n) || mem.get(&I.trup, n))
    return WQL3D_ENOMEM;
  T *sm = nullptr, *sp = nullptr;
  if (mem.get(&sm, 9 * n) || mem.get(&sp, 9 * n)) return WQL3D_ENOMEM;
  I.sat_m = sm;
  I.sat_p = sp;
  // trup starts at 1e9 (src/iface.f90); DS / DW start at 1e40 in the reference
  // and are multiplied by A(1) = 0 before first use, so zero is equivalent.
  std::vector<double> tr((size_t)n, 1.0e9);
  if (cudaMemcpyAsync(I.trup, tr.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s) != cudaSuccess)
    return WQL3D_ECUDA;
  const Blk<T> *bs[2] = {&b0, &b1};
  const std::vector<double> *cs[2] = {&coords0, &coords1};
  for (int side = 0; side < 2; ++side) {
    std::vector<double> t0, f, ra, nuc;
    const int face = side == 0 ? 1 : 0;
    const int xend = side == 0 ? b0.nx : 1;
    if (int rc = fault_maps<T>(desc, *bs[side], face, *cs[side], xend, t0, f, ra, nuc, s)) return rc;
    if (mem.get(&I.t0[side], 3 * n) || mem.get(&I.fs[side], n) || mem.get(&I.ra[side], n) || mem.get(&I.nuc[side], n))
      return WQL3D_ENOMEM;
    if (cudaMemcpyAsync(I.t0[side], t0.data(), sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(I.fs[side], f.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(I.ra[side], ra.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(I.nuc[side], nuc.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s) != cudaSuccess)
      return WQL3D_ECUDA;
    // the host vectors go out of scope at the end of this iteration
    if (cudaStreamSynchronize(s) != cudaSuccess) return WQL3D_ECUDA;
  }
  // the host vectors above go out of scope: finish the copies first
  if (cudaStreamSynchronize(s) != cudaSuccess) return WQL3D_ECUDA;
  // the one-process run initialises the state from block 1 (src/domain.f90:273)
  if (rs_problem(desc.fault_problem)) return rs_init_state<T>(I, b0, 1, coords0, b0.nx, s);
  return WQL3D_OK;
}

// Remote side: buffers, state and this side's prestress / strength map.
template <typename T, typename AllocT>
int setup_iface_remote(IfaceDev &I, const wql3d_domain_desc &desc, const Blk<T> &b, const std::vector<double> &coords,
                       int side, AllocT &mem, cudaStream_t s) {
  if (side != 1 && side != 2) return WQL3D_EINVAL;
  if (!fault_problem_ok(desc)) return WQL3D_EINVAL;
  const int ny = b.ny, nz = b.nz;
  const long long n = (long long)ny * nz;
  I.ny = ny;
  I.nz = nz;
  I.coupling = desc.coupling;
  I.serial = 0;
  fault_weakening(desc, &I.fd, &I.Dc);
  I.remote = side;
  if (mem.get(&I.S, 4 * n) || mem.get(&I.DS, 4 * n) || mem.get(&I.W, n) || mem.get(&I.DW, n) ||
      mem.get(&I.Svel, 3 * n) || mem.get(&I.Uhat, 6 * n) || mem.get(&I.Vhat, 6 * n) || mem.get(&I.trup, n))
    return WQL3D_ENOMEM;
  T *sat = nullptr, *snd = nullptr, *rcv = nullptr, *om = nullptr;
  if (mem.get(&sat, 9 * n) || mem.get(&snd, 9 * n) || mem.get(&rcv, 9 * n) || mem.get(&om, 3 * n))
    return WQL3D_ENOMEM;
  if (side == 1) I.sat_m = sat;
  else I.sat_p = sat;
  I.send = snd;
  I.recv = rcv;
  I.oppM = om;
  std::vector<double> tr((size_t)n, 1.0e9);
  if (cudaMemcpyAsync(I.trup, tr.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s) != cudaSuccess)
    return WQL3D_ECUDA;
  std::vector<double> t0, f, ra, nuc;
  const int xend = side == 1 ? b.nx : 1;
  if (int rc = fault_maps<T>(desc, b, side == 1 ? 1 : 0, coords, xend, t0, f, ra, nuc, s)) return rc;
  if (mem.get(&I.t0[side - 1], 3 * n) || mem.get(&I.fs[side - 1], n) || mem.get(&I.ra[side - 1], n) ||
      mem.get(&I.nuc[side - 1], n))
    return WQL3D_ENOMEM;
  if (cudaMemcpyAsync(I.t0[side - 1], t0.data(), sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(I.fs[side - 1], f.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(I.ra[side - 1], ra.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(I.nuc[side - 1], nuc.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s) != cudaSuccess)
    return WQL3D_ECUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return WQL3D_ECUDA;
  // one block per rank: each rank initialises the state from its own face
  // (src/domain.f90:273-274)
  if (rs_problem(desc.fault_problem)) return rs_init_state<T>(I, b, side == 1 ? 1 : 0, coords, xend, s);
  return WQL3D_OK;
}

// ---------------------------------------------------------------------------
// per-point interface law in the (n, m, l) basis
// ---------------------------------------------------------------------------
struct IfacePoint {
  double p[3], q[3], phi[3], eta_p, eta_s;
};

__device__ __forceinline__ void iface_characteristics(const double *U, const double *V, double Z1s, double Z2s,
                                                      double Z1p, double Z2p, IfacePoint &c) {
  // common head of Welded_Interface / Linear_Friction / Slip_Weakening_Friction
  c.p[0] = __dsub_rn(__dmul_rn(Z1p, U[0]), U[3]);
  c.p[1] = __dsub_rn(__dmul_rn(Z1s, U[1]), U[4]);
  c.p[2] = __dsub_rn(__dmul_rn(Z1s, U[2]), U[5]);
  c.q[0] = __dadd_rn(__dmul_rn(Z2p, V[0]), V[3]);
  c.q[1] = __dadd_rn(__dmul_rn(Z2s, V[1]), V[4]);
  c.q[2] = __dadd_rn(__dmul_rn(Z2s, V[2]), V[5]);
  c.eta_p = 1.0 / (1.0 / Z1p + 1.0 / Z2p);
  c.eta_s = 1.0 / (1.0 / Z1s + 1.0 / Z2s);
  c.phi[0] = __dmul_rn(c.eta_p, __dsub_rn(c.q[0] / Z2p, c.p[0] / Z1p));
  c.phi[1] = __dmul_rn(c.eta_s, __dsub_rn(c.q[1] / Z2s, c.p[1] / Z1s));
  c.phi[2] = __dmul_rn(c.eta_s, __dsub_rn(c.q[2] / Z2s, c.p[2] / Z1s));
}

__device__ __forceinline__ double dot3(const double a[3], const double b[3]) {
  return __dadd_rn(__dadd_rn(__dmul_rn(a[0], b[0]), __dmul_rn(a[1], b[1])), __dmul_rn(a[2], b[2]));
}

// TPV101 / TPV102 prestress in the face basis at time t: the initial stress
// (-120, 0, -120, 0, 75, 0) of src/initial_stress_condition.f90:114-120 as
// tractions on n, rotated onto n, m, l, plus the nucleation 25 F(r) G(t) on
// T0_l (src/Interface_Condition.f90:2324-2385)
__device__ __forceinline__ void rs_prestress(double t, double nuc, const double n[3], const double m[3],
                                             const double l[3], double T0[3]) {
  const double sxx = -120.0, syy = 0.0, szz = -120.0, sxy = 0.0, sxz = 75.0, syz = 0.0;
  const double Tx = __dadd_rn(__dadd_rn(__dmul_rn(n[0], sxx), __dmul_rn(n[1], sxy)), __dmul_rn(n[2], sxz));
  const double Ty = __dadd_rn(__dadd_rn(__dmul_rn(n[0], sxy), __dmul_rn(n[1], syy)), __dmul_rn(n[2], syz));
  const double Tz = __dadd_rn(__dadd_rn(__dmul_rn(n[0], sxz), __dmul_rn(n[1], syz)), __dmul_rn(n[2], szz));
  const double Tv[3] = {Tx, Ty, Tz};
  T0[0] = dot3(n, Tv);
  T0[1] = dot3(m, Tv);
  T0[2] = dot3(l, Tv);
  double G = 0.0;
  if (t > 0.0 && t < 1.0) G = exp(__dmul_rn(__dsub_rn(t, 1.0), __dsub_rn(t, 1.0)) / __dmul_rn(t, __dsub_rn(t, 2.0)));
  if (t >= 1.0) G = 1.0;
  T0[2] = __dadd_rn(T0[2], __dmul_rn(nuc, G));
}

// f(V) = V + a sigma_n / eta asinh(V / (2 V0) exp(psi / a)) - Phi / eta
// (src/Interface_Condition.f90:1242-1263)
__device__ __forceinline__ double rs_f(double V, double Phi, double eta, double sn, double psi, double a) {
  const double g = asinh(__dmul_rn(__dmul_rn(0.5, V) / kRsV0, exp(psi / a)));
  return __dsub_rn(__dadd_rn(V, __dmul_rn(__dmul_rn(a, sn) / eta, g)), Phi / eta);
}

// Regula_Falsi, src/Interface_Condition.f90:1170-1239: bracket [0, Phi/eta],
// absolute tolerance 1e-12, at most 5000 iterations (the reference's cap)
__device__ double rs_regula_falsi(double V, double Phi, double eta, double sn, double psi, double a) {
  const double tol = 1.0e-12;
  double Vl = 0.0, Vr = Phi / eta;
  double fv = rs_f(V, Phi, eta, sn, psi, a);
  double fl = rs_f(Vl, Phi, eta, sn, psi, a);
  double fr = rs_f(Vr, Phi, eta, sn, psi, a);
  if (fabs(fv) <= tol) return V;
  if (fabs(fl) <= tol) return Vl;
  if (fabs(fr) <= tol) return Vr;
  double err = 1.0;
  for (int k = 1; k <= 5000 && err >= tol; ++k) {
    const double V1 = V;
    if (__dmul_rn(fv, fl) > tol) {
      Vl = V;
      V = __dsub_rn(Vr, __dmul_rn(__dsub_rn(Vr, Vl), fr) / __dsub_rn(fr, fl));
      fl = fv;
    } else if (__dmul_rn(fv, fr) > tol) {
      Vr = V;
      V = __dsub_rn(Vr, __dmul_rn(__dsub_rn(Vr, Vl), fr) / __dsub_rn(fr, fl));
      fr = fv;
    }
    fv = rs_f(V, Phi, eta, sn, psi, a);
    err = fabs(__dsub_rn(V, V1));
  }
  return V;
}

// Interface law at one point: P (side-1 hats) and Q (side-2 hats) from the
// rotated traces U, V.  T0 / fs: this side's prestress and static friction;
// rate-and-state: psi the state, ra the direct-effect parameter, *Vrs the
// solved slip rate (the state-rate input).
__device__ void iface_law(const IfaceDev &I, const double *U, const double *V, double Z1s, double Z2s, double Z1p,
                          double Z2p, const double T0[3], double fsk, double slip, double psi, double ra,
                          double *Vrs, double *P, double *Q) {
  IfacePoint c;
  iface_characteristics(U, V, Z1s, Z2s, Z1p, Z2p, c);
  P[0] = __dsub_rn(c.q[0], c.phi[0]) / Z2p;
  P[3] = c.phi[0];
  Q[0] = __dadd_rn(c.p[0], c.phi[0]) / Z1p;
  Q[3] = c.phi[0];
  if (I.coupling == WQL3D_IFACE_RATE_STATE) {
    // rate_state_friction + solve('rate-and-state_friction'),
    // src/Interface_Condition.f90:918-1067, 1095-1168
    const double T0n = T0[0], T0m = T0[1], T0l = T0[2];
    const double sigma_n = fmax(0.0, -__dadd_rn(T0n, c.phi[0]));
    double vm = __dsub_rn(V[1], U[1]), vl = __dsub_rn(V[2], U[2]);
    const double phi1 = __dadd_rn(T0m, c.phi[1]), phi2 = __dadd_rn(T0l, c.phi[2]);
    const double Phi = sqrt(__dadd_rn(__dmul_rn(phi1, phi1), __dmul_rn(phi2, phi2)));
    double Vs = sqrt(__dadd_rn(__dmul_rn(vm, vm), __dmul_rn(vl, vl)));
    if (Vs > Phi) Vs = __dmul_rn(0.5, Phi) / c.eta_s;
    Vs = rs_regula_falsi(Vs, Phi, c.eta_s, sigma_n, psi, ra);
    const double fv = __dmul_rn(__dmul_rn(sigma_n, ra), asinh(__dmul_rn(__dmul_rn(0.5, Vs) / kRsV0, exp(psi / ra))));
    const double den = __dadd_rn(c.eta_s, fv / Vs);
    vm = phi1 / den;
    vl = phi2 / den;
    const double tm = __dsub_rn(__dsub_rn(phi1, __dmul_rn(c.eta_s, vm)), T0m);
    const double tl = __dsub_rn(__dsub_rn(phi2, __dmul_rn(c.eta_s, vl)), T0l);
    Q[1] = __dadd_rn(__dadd_rn(tm, c.p[1]) / Z1s, vm);
    Q[2] = __dadd_rn(__dadd_rn(tl, c.p[2]) / Z1s, vl);
    P[1] = __dsub_rn(__dsub_rn(c.q[1], tm) / Z2s, vm);
    P[2] = __dsub_rn(__dsub_rn(c.q[2], tl) / Z2s, vl);
    P[4] = tm; P[5] = tl; Q[4] = tm; Q[5] = tl;
    *Vrs = Vs;
  } else if (I.coupling == WQL3D_IFACE_SLIP_WEAKENING) {
    // Slip_Weakening_Friction + solve('slip-weakening_friction'),
    // src/Interface_Condition.f90:745-916, 1095-1168
    const double T0n = T0[0], T0m = T0[1], T0l = T0[2];
    const double al = __dadd_rn(T0l, c.phi[2]), am = __dadd_rn(T0m, c.phi[1]);
    const double tau_lock = sqrt(__dadd_rn(__dmul_rn(al, al), __dmul_rn(am, am)));
    const double sigma_n = fmax(0.0, -__dadd_rn(T0n, c.phi[0]));
    // Tau_strength: f = fs - (fs - fd) min(D, Dc) / Dc
    const double f = __dsub_rn(fsk, __dmul_rn(__dsub_rn(fsk, I.fd), fmin(slip, I.Dc)) / I.Dc);
    const double tau_str = __dmul_rn(sigma_n, f);
    double tm, tl, vm, vl;
    if (tau_lock > tau_str) {
      const double phi1 = am, phi2 = al;
      const double Phi = sqrt(__dadd_rn(__dmul_rn(phi1, phi1), __dmul_rn(phi2, phi2)));
      const double Vs = __dsub_rn(Phi, tau_str) / c.eta_s;
      const double den = __dadd_rn(c.eta_s, tau_str / Vs);
      vm = phi1 / den;
      vl = phi2 / den;
      tm = __dsub_rn(__dsub_rn(phi1, __dmul_rn(c.eta_s, vm)), T0m);
      tl = __dsub_rn(__dsub_rn(phi2, __dmul_rn(c.eta_s, vl)), T0l);
    } else {
      tm = c.phi[1];
      tl = c.phi[2];
      vm = 0.0;
      vl = 0.0;
    }
    Q[1] = __dadd_rn(__dadd_rn(tm, c.p[1]) / Z1s, vm);
    Q[2] = __dadd_rn(__dadd_rn(tl, c.p[2]) / Z1s, vl);
    P[1] = __dsub_rn(__dsub_rn(c.q[1], tm) / Z2s, vm);
    P[2] = __dsub_rn(__dsub_rn(c.q[2], tl) / Z2s, vl);
    P[4] = tm; P[5] = tl; Q[4] = tm; Q[5] = tl;
  } else if (I.coupling == WQL3D_IFACE_LINEAR) {
    // Linear_Friction with alpha = 1e14, src/Interface_Condition.f90:601-741
    // (the reference leaves u_out(2) unassigned; it is set to u_m_hat here)
    const double alpha = 1.0e14;
    const double ae = __dadd_rn(alpha, c.eta_s);
    const double tm = __dmul_rn(alpha / ae, c.phi[1]);
    const double tl = __dmul_rn(alpha / ae, c.phi[2]);
    P[4] = tm; P[5] = tl; Q[4] = tm; Q[5] = tl;
    Q[1] = __dadd_rn(__dadd_rn(c.p[1], tm) / Z1s, __dmul_rn(1.0 / ae, c.phi[1]));
    Q[2] = __dadd_rn(__dadd_rn(c.p[2], tl) / Z1s, __dmul_rn(1.0 / ae, c.phi[2]));
    P[1] = __dsub_rn(__dsub_rn(c.q[1], tm) / Z2s, __dmul_rn(1.0 / ae, c.phi[1]));
    P[2] = __dsub_rn(__dsub_rn(c.q[2], tl) / Z2s, __dmul_rn(1.0 / ae, c.phi[2]));
  } else {
    // Welded_Interface, src/Interface_Condition.f90:504-598
    P[2] = __dsub_rn(c.q[2], c.phi[2]) / Z2s; P[5] = c.phi[2];
    Q[2] = __dadd_rn(c.p[2], c.phi[2]) / Z1s; Q[5] = c.phi[2];
    P[1] = __dsub_rn(c.q[1], c.phi[1]) / Z2s; P[4] = c.phi[1];
    Q[1] = __dadd_rn(c.p[1], c.phi[1]) / Z1s; Q[4] = c.phi[1];
  }
}

__device__ __forceinline__ void rot_in(double *w, const double n[3], const double m[3], const double l[3]) {
  // Rotate_in_Local_Cordinates, src/CouplingForcing.f90:466-520
  const double a[6] = {w[0], w[1], w[2], w[3], w[4], w[5]};
  w[0] = dot3(n, a);
  w[1] = dot3(m, a);
  w[2] = dot3(l, a);
  w[3] = dot3(n, a + 3);
  w[4] = dot3(m, a + 3);
  w[5] = dot3(l, a + 3);
}

__device__ __forceinline__ void rot_back(double *w, const double n[3], const double m[3], const double l[3]) {
  // Rotate_Back_Physical_Cordinates, src/CouplingForcing.f90:524-580
  const double a[6] = {w[0], w[1], w[2], w[3], w[4], w[5]};
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    w[i] = __dadd_rn(__dadd_rn(__dmul_rn(n[i], a[0]), __dmul_rn(m[i], a[1])), __dmul_rn(l[i], a[2]));
    w[3 + i] = __dadd_rn(__dadd_rn(__dmul_rn(n[i], a[3]), __dmul_rn(m[i], a[4])), __dmul_rn(l[i], a[5]));
  }
}

// SAT vector of one side from grid (g) and hat (h) values in x, y, z
// components, src/CouplingForcing.f90:250-437 (side 1: p = (Z u + T)/2 with
// block 1's impedances; side 2: q = (Z v - T)/2 with block 2's, stress rows
// negated).
__device__ void iface_sat(int side, const double *g, const double *h, double lam, double mu, double rho,
                          const double n[3], const double m[3], const double l[3], double qx, double qy,
                          double qz, double *out) {
  const double c_p = sqrt(__dadd_rn(__dmul_rn(2.0, mu), lam) / rho), c_s = sqrt(mu / rho);
  const double Zp = __dmul_rn(rho, c_p), Zs = __dmul_rn(rho, c_s);
  const double norm = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(qx, qx), __dmul_rn(qy, qy)), __dmul_rn(qz, qz)));
  const double *e[3] = {n, m, l};
  double Mz[3][3], Mi[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      Mz[i][j] = __dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(e[i][0], e[j][0]), Zp), __dmul_rn(__dmul_rn(e[i][1], e[j][1]), Zs)),
                           __dmul_rn(__dmul_rn(e[i][2], e[j][2]), Zs));
      Mi[i][j] = __dadd_rn(__dadd_rn(__dmul_rn(e[i][0], e[j][0]) / Zp, __dmul_rn(e[i][1], e[j][1]) / Zs),
                           __dmul_rn(e[i][2], e[j][2]) / Zs);
    }
  double dch[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    double sh = __dadd_rn(__dadd_rn(__dmul_rn(Mz[i][0], h[0]), __dmul_rn(Mz[i][1], h[1])), __dmul_rn(Mz[i][2], h[2]));
    double sg = __dadd_rn(__dadd_rn(__dmul_rn(Mz[i][0], g[0]), __dmul_rn(Mz[i][1], g[1])), __dmul_rn(Mz[i][2], g[2]));
    sh = side == 1 ? __dadd_rn(sh, h[3 + i]) : __dsub_rn(sh, h[3 + i]);
    sg = side == 1 ? __dadd_rn(sg, g[3 + i]) : __dsub_rn(sg, g[3 + i]);
    dch[i] = __dsub_rn(__dmul_rn(0.5, sg), __dmul_rn(0.5, sh));
  }
  double r[3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
    r[i] = __dadd_rn(__dadd_rn(__dmul_rn(Mi[i][0], dch[0]), __dmul_rn(Mi[i][1], dch[1])), __dmul_rn(Mi[i][2], dch[2]));
  const double l2m = __dadd_rn(__dmul_rn(2.0, mu), lam);
  const double nr = norm / rho;
#pragma unroll
  for (int i = 0; i < 3; ++i) out[i] = __dmul_rn(nr, dch[i]);
  double s3 = __dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(l2m, qx), r[0]), __dmul_rn(__dmul_rn(lam, qy), r[1])), __dmul_rn(__dmul_rn(lam, qz), r[2]));
  double s4 = __dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(l2m, qy), r[1]), __dmul_rn(__dmul_rn(lam, qz), r[2])), __dmul_rn(__dmul_rn(lam, qx), r[0]));
  double s5 = __dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(l2m, qz), r[2]), __dmul_rn(__dmul_rn(lam, qy), r[1])), __dmul_rn(__dmul_rn(lam, qx), r[0]));
  double s6 = __dmul_rn(mu, __dadd_rn(__dmul_rn(qy, r[0]), __dmul_rn(qx, r[1])));
  double s7 = __dmul_rn(mu, __dadd_rn(__dmul_rn(qz, r[0]), __dmul_rn(qx, r[2])));
  double s8 = __dmul_rn(mu, __dadd_rn(__dmul_rn(qz, r[1]), __dmul_rn(qy, r[2])));
  const double sg = side == 1 ? 1.0 : -1.0;
  out[3] = sg * s3; out[4] = sg * s4; out[5] = sg * s5;
  out[6] = sg * s6; out[7] = sg * s7; out[8] = sg * s8;
}

template <typename T>
__global__ void __launch_bounds__(128) k_iface(Blk<T> b0, Blk<T> b1, IfaceDev I, StageArgs a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = I.ny * I.nz;
  if (k >= n) return;
  const int y = k % I.ny + 1, z = k / I.ny + 1;
  const T *F0 = a.cur ? b0.F1 : b0.F0;
  const T *F1 = a.cur ? b1.F1 : b1.F0;
  const long long p0 = pidx(b0, b0.nx, y, z), p1 = pidx(b1, 1, y, z);
  double uF[9], vF[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    uF[c] = (double)F0[c * b0.vol + p0];
    vF[c] = (double)F1[c * b1.vol + p1];
  }
  const double lam1 = (double)b0.M[p0], mu1 = (double)b0.M[b0.vol + p0], rho1 = (double)b0.M[2 * b0.vol + p0];
  const double lam2 = (double)b1.M[p1], mu2 = (double)b1.M[b1.vol + p1], rho2 = (double)b1.M[2 * b1.vol + p1];
  const double c1p = sqrt(__dadd_rn(__dmul_rn(2.0, mu1), lam1) / rho1), c1s = sqrt(mu1 / rho1);
  const double c2p = sqrt(__dadd_rn(__dmul_rn(2.0, mu2), lam2) / rho2), c2s = sqrt(mu2 / rho2);
  const double Z1s = __dmul_rn(rho1, c1s), Z2s = __dmul_rn(rho2, c2s);
  const double Z1p = __dmul_rn(rho1, c1p), Z2p = __dmul_rn(rho2, c2p);

  double ds[4], S4;
  if (a.flags & F_ISAT) {
    S4 = I.S[3 * n + k];
#pragma unroll
    for (int c = 0; c < 4; ++c) ds[c] = I.DS[c * n + k];
    double dw = I.DW[k];
    if (a.flags & F_SCALE) {
#pragma unroll
      for (int c = 0; c < 4; ++c) ds[c] = __dmul_rn(a.A, ds[c]);
      dw = __dmul_rn(a.A, dw);
    }
    // stage time of the interface law (D%t at enforce_bound_iface_conditions)
    const double ts = a.stage <= 1 ? a.time->t : a.time->t + c_rkC[a.stage - 1] * a.dt;
    const bool rs = I.coupling == WQL3D_IFACE_RATE_STATE;
    for (int side = 1; side <= 2; ++side) {
      const Blk<T> &b = side == 1 ? b0 : b1;
      const long long p = side == 1 ? p0 : p1;
      const T *B = b.nrm[side == 1 ? 1 : 0];   // face basis l(3) m(3) n(3), face-local (y, z)
      double n3[3], m3[3], l3[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        l3[c] = (double)B[(0 + c) * n + k];
        m3[c] = (double)B[(3 + c) * n + k];
        n3[c] = (double)B[(6 + c) * n + k];
      }
      // tractions T = sigma n and velocities, src/CouplingForcing.f90:99-165
      double u[6], v[6];
      u[0] = uF[0]; u[1] = uF[1]; u[2] = uF[2];
      v[0] = vF[0]; v[1] = vF[1]; v[2] = vF[2];
      {
        const double su[3] = {uF[3], uF[6], uF[7]}, su2[3] = {uF[6], uF[4], uF[8]}, su3[3] = {uF[7], uF[8], uF[5]};
        const double sv[3] = {vF[3], vF[6], vF[7]}, sv2[3] = {vF[6], vF[4], vF[8]}, sv3[3] = {vF[7], vF[8], vF[5]};
        u[3] = dot3(n3, su); u[4] = dot3(n3, su2); u[5] = dot3(n3, su3);
        v[3] = dot3(n3, sv); v[4] = dot3(n3, sv2); v[5] = dot3(n3, sv3);
      }
      rot_in(u, n3, m3, l3);
      rot_in(v, n3, m3, l3);
      double T0[3] = {I.t0[side - 1][k], I.t0[side - 1][n + k], I.t0[side - 1][2 * n + k]};
      if (rs) rs_prestress(ts, I.nuc[side - 1][k], n3, m3, l3, T0);
      double P[6], Q[6], Vrs = 0.0;
      iface_law(I, u, v, Z1s, Z2s, Z1p, Z2p, T0, I.fs[side - 1][k], S4, I.W[k], rs ? I.ra[side - 1][k] : 1.0, &Vrs,
                P, Q);
      const double Vel = sqrt(__dadd_rn(__dmul_rn(__dsub_rn(Q[1], P[1]), __dsub_rn(Q[1], P[1])),
                                        __dmul_rn(__dsub_rn(Q[2], P[2]), __dsub_rn(Q[2], P[2]))));
      if (side == 1 || I.serial) {
#pragma unroll
        for (int c = 0; c < 3; ++c) ds[c] = __dsub_rn(__dadd_rn(ds[c], Q[c]), P[c]);
        ds[3] = __dadd_rn(ds[3], Vel);
        // rate of state, TPV101 / TPV102 (src/Interface_Condition.f90:431-436)
        if (rs)
          dw = __dsub_rn(__dadd_rn(dw, __dmul_rn(kRsB * kRsV0 / kRsL0, exp(-__dsub_rn(I.W[k], kRsF0) / kRsB))),
                         __dmul_rn(Vrs, kRsB) / kRsL0);
      }
      if (a.stage == 1 && (side == 1 || I.serial)) {
        // fault outputs, src/Interface_Condition.f90:470-486 and
        // src/CouplingForcing.f90:203-215 (components 1:3 = v_hat - u_hat)
        const double Tn = I.coupling == WQL3D_IFACE_LOCKED ? 0.0 : T0[0];
        const double Tm = I.coupling == WQL3D_IFACE_LOCKED ? 0.0 : T0[1];
        const double Tl = I.coupling == WQL3D_IFACE_LOCKED ? 0.0 : T0[2];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const double sv = __dsub_rn(Q[c], P[c]);
          I.Uhat[c * n + k] = sv;
          I.Vhat[c * n + k] = sv;
          I.Svel[c * n + k] = sv;
        }
        I.Uhat[3 * n + k] = __dadd_rn(P[3], Tn); I.Vhat[3 * n + k] = __dadd_rn(Q[3], Tn);
        I.Uhat[4 * n + k] = __dadd_rn(P[4], Tm); I.Vhat[4 * n + k] = __dadd_rn(Q[4], Tm);
        I.Uhat[5 * n + k] = __dadd_rn(P[5], Tl); I.Vhat[5 * n + k] = __dadd_rn(Q[5], Tl);
        // rupture_front, src/CouplingForcing.f90:583-600
        const double s1 = __dsub_rn(Q[1], P[1]), s2 = __dsub_rn(Q[2], P[2]);
        if (sqrt(__dadd_rn(__dmul_rn(s1, s1), __dmul_rn(s2, s2))) > 1.0e-3) I.trup[k] = fmin(I.trup[k], a.time->t);
      }
      rot_back(u, n3, m3, l3);
      rot_back(v, n3, m3, l3);
      rot_back(P, n3, m3, l3);
      rot_back(Q, n3, m3, l3);
      // metric of the calling block at its interface face (q1 = q2)
      const double qx = (double)b.met[(long long)0 * b.vol + p];
      const double qy = (double)b.met[(long long)3 * b.vol + p];
      const double qz = (double)b.met[(long long)6 * b.vol + p];
      double sat[9];
      if (side == 1) iface_sat(1, u, P, lam1, mu1, rho1, n3, m3, l3, qx, qy, qz, sat);
      else iface_sat(2, v, Q, lam2, mu2, rho2, n3, m3, l3, qx, qy, qz, sat);
      T *out = (T *)(side == 1 ? I.sat_m : I.sat_p);
#pragma unroll
      for (int c = 0; c < 9; ++c) out[c * n + k] = (T)sat[c];
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) I.DS[c * n + k] = ds[c];
    I.DW[k] = dw;
  }
  if (a.flags & F_UPDATE) {
    // update_fields for the interface (src/iface.f90): S = S + B dt DS
#pragma unroll
    for (int c = 0; c < 4; ++c) I.S[c * n + k] = __dadd_rn(I.S[c * n + k], __dmul_rn(a.Bdt, I.DS[c * n + k]));
    I.W[k] = __dadd_rn(I.W[k], __dmul_rn(a.Bdt, I.DW[k]));
  }
}

__global__ void k_iface_scale(IfaceDev I, double A) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = I.ny * I.nz;
  if (k >= n) return;
#pragma unroll
  for (int c = 0; c < 4; ++c) I.DS[c * n + k] = __dmul_rn(A, I.DS[c * n + k]);
  I.DW[k] = __dmul_rn(A, I.DW[k]);
}

// this block's interface face trace into the send buffer (copy_fields_to_boundary,
// src/block.f90:466-482)
template <typename T>
__global__ void k_pack_face(Blk<T> b, int cur, int side, T *send) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = b.ny * b.nz;
  if (k >= n) return;
  const int y = k % b.ny + 1, z = k / b.ny + 1;
  const T *F = cur ? b.F1 : b.F0;
  const long long p = pidx(b, side == 1 ? b.nx : 1, y, z);
#pragma unroll
  for (int c = 0; c < 9; ++c) send[c * n + k] = F[c * b.vol + p];
}

// One side of the interface (the other block lives in another process): the
// same law, outputs and SAT vector as k_iface's side I.remote, with the
// other side's trace and material from recv / oppM.  Each process keeps its
// own slip state and adds to it once per stage (src/domain.f90:615-644 on
// one rank per block).
template <typename T>
__global__ void __launch_bounds__(128) k_iface_remote(Blk<T> b, IfaceDev I, StageArgs a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = I.ny * I.nz;
  if (k >= n) return;
  const int side = I.remote;
  if (a.flags & F_ISAT) {
    const int y = k % I.ny + 1, z = k / I.ny + 1;
    const T *F = a.cur ? b.F1 : b.F0;
    const long long p = pidx(b, side == 1 ? b.nx : 1, y, z);
    const T *R = (const T *)I.recv;
    const T *OM = (const T *)I.oppM;
    double own[9], opp[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) {
      own[c] = (double)F[c * b.vol + p];
      opp[c] = (double)R[c * n + k];
    }
    const double *uF = side == 1 ? own : opp;
    const double *vF = side == 1 ? opp : own;
    const double lo = (double)b.M[p], mo = (double)b.M[b.vol + p], ro = (double)b.M[2 * b.vol + p];
    const double lr = (double)OM[k], mr = (double)OM[n + k], rr = (double)OM[2 * n + k];
    const double lam1 = side == 1 ? lo : lr, mu1 = side == 1 ? mo : mr, rho1 = side == 1 ? ro : rr;
    const double lam2 = side == 1 ? lr : lo, mu2 = side == 1 ? mr : mo, rho2 = side == 1 ? rr : ro;
    const double c1p = sqrt(__dadd_rn(__dmul_rn(2.0, mu1), lam1) / rho1), c1s = sqrt(mu1 / rho1);
    const double c2p = sqrt(__dadd_rn(__dmul_rn(2.0, mu2), lam2) / rho2), c2s = sqrt(mu2 / rho2);
    const double Z1s = __dmul_rn(rho1, c1s), Z2s = __dmul_rn(rho2, c2s);
    const double Z1p = __dmul_rn(rho1, c1p), Z2p = __dmul_rn(rho2, c2p);
    const double S4 = I.S[3 * n + k];
    double ds[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      ds[c] = I.DS[c * n + k];
      if (a.flags & F_SCALE) ds[c] = __dmul_rn(a.A, ds[c]);
    }
    double dw = I.DW[k];
    if (a.flags & F_SCALE) dw = __dmul_rn(a.A, dw);
    const double ts = a.stage <= 1 ? a.time->t : a.time->t + c_rkC[a.stage - 1] * a.dt;
    const bool rs = I.coupling == WQL3D_IFACE_RATE_STATE;
    const T *B = b.nrm[side == 1 ? 1 : 0];
    double n3[3], m3[3], l3[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      l3[c] = (double)B[(0 + c) * n + k];
      m3[c] = (double)B[(3 + c) * n + k];
      n3[c] = (double)B[(6 + c) * n + k];
    }
    double u[6], v[6];
    u[0] = uF[0]; u[1] = uF[1]; u[2] = uF[2];
    v[0] = vF[0]; v[1] = vF[1]; v[2] = vF[2];
    {
      const double su[3] = {uF[3], uF[6], uF[7]}, su2[3] = {uF[6], uF[4], uF[8]}, su3[3] = {uF[7], uF[8], uF[5]};
      const double sv[3] = {vF[3], vF[6], vF[7]}, sv2[3] = {vF[6], vF[4], vF[8]}, sv3[3] = {vF[7], vF[8], vF[5]};
      u[3] = dot3(n3, su); u[4] = dot3(n3, su2); u[5] = dot3(n3, su3);
      v[3] = dot3(n3, sv); v[4] = dot3(n3, sv2); v[5] = dot3(n3, sv3);
    }
    rot_in(u, n3, m3, l3);
    rot_in(v, n3, m3, l3);
    double T0[3] = {I.t0[side - 1][k], I.t0[side - 1][n + k], I.t0[side - 1][2 * n + k]};
    if (rs) rs_prestress(ts, I.nuc[side - 1][k], n3, m3, l3, T0);
    double P[6], Q[6], Vrs = 0.0;
    iface_law(I, u, v, Z1s, Z2s, Z1p, Z2p, T0, I.fs[side - 1][k], S4, I.W[k], rs ? I.ra[side - 1][k] : 1.0, &Vrs, P,
              Q);
    const double Vel = sqrt(__dadd_rn(__dmul_rn(__dsub_rn(Q[1], P[1]), __dsub_rn(Q[1], P[1])),
                                      __dmul_rn(__dsub_rn(Q[2], P[2]), __dsub_rn(Q[2], P[2]))));
#pragma unroll
    for (int c = 0; c < 3; ++c) ds[c] = __dsub_rn(__dadd_rn(ds[c], Q[c]), P[c]);
    ds[3] = __dadd_rn(ds[3], Vel);
    if (rs)
      dw = __dsub_rn(__dadd_rn(dw, __dmul_rn(kRsB * kRsV0 / kRsL0, exp(-__dsub_rn(I.W[k], kRsF0) / kRsB))),
                     __dmul_rn(Vrs, kRsB) / kRsL0);
    if (a.stage == 1) {
      const double Tn = I.coupling == WQL3D_IFACE_LOCKED ? 0.0 : T0[0];
      const double Tm = I.coupling == WQL3D_IFACE_LOCKED ? 0.0 : T0[1];
      const double Tl = I.coupling == WQL3D_IFACE_LOCKED ? 0.0 : T0[2];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double sv = __dsub_rn(Q[c], P[c]);
        I.Uhat[c * n + k] = sv;
        I.Vhat[c * n + k] = sv;
        I.Svel[c * n + k] = sv;
      }
      I.Uhat[3 * n + k] = __dadd_rn(P[3], Tn); I.Vhat[3 * n + k] = __dadd_rn(Q[3], Tn);
      I.Uhat[4 * n + k] = __dadd_rn(P[4], Tm); I.Vhat[4 * n + k] = __dadd_rn(Q[4], Tm);
      I.Uhat[5 * n + k] = __dadd_rn(P[5], Tl); I.Vhat[5 * n + k] = __dadd_rn(Q[5], Tl);
      const double s1 = __dsub_rn(Q[1], P[1]), s2 = __dsub_rn(Q[2], P[2]);
      if (sqrt(__dadd_rn(__dmul_rn(s1, s1), __dmul_rn(s2, s2))) > 1.0e-3) I.trup[k] = fmin(I.trup[k], a.time->t);
    }
    rot_back(u, n3, m3, l3);
    rot_back(v, n3, m3, l3);
    rot_back(P, n3, m3, l3);
    rot_back(Q, n3, m3, l3);
    const double qx = (double)b.met[(long long)0 * b.vol + p];
    const double qy = (double)b.met[(long long)3 * b.vol + p];
    const double qz = (double)b.met[(long long)6 * b.vol + p];
    double sat[9];
    if (side == 1) iface_sat(1, u, P, lam1, mu1, rho1, n3, m3, l3, qx, qy, qz, sat);
    else iface_sat(2, v, Q, lam2, mu2, rho2, n3, m3, l3, qx, qy, qz, sat);
    T *out = (T *)(side == 1 ? I.sat_m : I.sat_p);
#pragma unroll
    for (int c = 0; c < 9; ++c) out[c * n + k] = (T)sat[c];
#pragma unroll
    for (int c = 0; c < 4; ++c) I.DS[c * n + k] = ds[c];
    I.DW[k] = dw;
  }
  if (a.flags & F_UPDATE) {
#pragma unroll
    for (int c = 0; c < 4; ++c) I.S[c * n + k] = __dadd_rn(I.S[c * n + k], __dmul_rn(a.Bdt, I.DS[c * n + k]));
    I.W[k] = __dadd_rn(I.W[k], __dmul_rn(a.Bdt, I.DW[k]));
  }
}

template <typename T>
void launch_iface(IfaceDev &I, const Blk<T> &b0, const Blk<T> &b1, const StageArgs &a, cudaStream_t s) {
  const int n = I.ny * I.nz;
  if (I.remote) k_iface_remote<T><<<(n + 127) / 128, 128, 0, s>>>(b0, I, a);
  else k_iface<T><<<(n + 127) / 128, 128, 0, s>>>(b0, b1, I, a);
}

template <typename T>
void launch_iface_update(IfaceDev &I, const Blk<T> &b0, const Blk<T> &b1, double Bdt, cudaStream_t s) {
  StageArgs a;
  a.cur = 0;
  a.flags = F_UPDATE;
  a.stage = 0;
  a.A = 1.0;
  a.Bdt = Bdt;
  a.dt = 0.0;
  a.time = nullptr;
  const int n = I.ny * I.nz;
  if (I.remote) k_iface_remote<T><<<(n + 127) / 128, 128, 0, s>>>(b0, I, a);
  else k_iface<T><<<(n + 127) / 128, 128, 0, s>>>(b0, b1, I, a);
}

// this block's face material (lambda, mu, rho) into a 3 x n device buffer
template <typename T>
__global__ void k_pack_face_material(Blk<T> b, int side, T *out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = b.ny * b.nz;
  if (k >= n) return;
  const int y = k % b.ny + 1, z = k / b.ny + 1;
  const long long p = pidx(b, side == 1 ? b.nx : 1, y, z);
#pragma unroll
  for (int c = 0; c < 3; ++c) out[c * n + k] = b.M[c * b.vol + p];
}

inline void iface_scale(IfaceDev &I, double A, cudaStream_t s) {
  const int n = I.ny * I.nz;
  k_iface_scale<<<(n + 127) / 128, 128, 0, s>>>(I, A);
}

// per point S(4) W Svel(|m,l| slip rate at stage 1) trup, like the oracle's orc_get_iface
inline int iface_download(IfaceDev &I, double *out, cudaStream_t s) {
  const long long n = (long long)I.ny * I.nz;
  std::vector<double> S((size_t)(4 * n)), W((size_t)n), V((size_t)(3 * n)), tr((size_t)n);
  if (cudaMemcpyAsync(S.data(), I.S, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(W.data(), I.W, sizeof(double) * n, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(V.data(), I.Svel, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(tr.data(), I.trup, sizeof(double) * n, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return WQL3D_ECUDA;
  for (long long k = 0; k < n; ++k) {
    for (int c = 0; c < 4; ++c) out[7 * k + c] = S[(size_t)(c * n + k)];
    out[7 * k + 4] = W[(size_t)k];
    out[7 * k + 5] = std::sqrt(V[(size_t)(n + k)] * V[(size_t)(n + k)] + V[(size_t)(2 * n + k)] * V[(size_t)(2 * n + k)]);
    out[7 * k + 6] = tr[(size_t)k];
  }
  return WQL3D_OK;
}

// one fault output (WQL3D_FO_*), layout [component][z][y]
inline int iface_fault_output(IfaceDev &I, int kind, double *out, cudaStream_t s) {
  const long long n = (long long)I.ny * I.nz;
  const double *src = nullptr;
  int nc = 0;
  switch (kind) {
    case WQL3D_FO_S: src = I.S; nc = 4; break;
    case WQL3D_FO_SVEL: src = I.Svel; nc = 3; break;
    case WQL3D_FO_UHAT: src = I.Uhat; nc = 6; break;
    case WQL3D_FO_VHAT: src = I.Vhat; nc = 6; break;
    case WQL3D_FO_STATE: src = I.W; nc = 1; break;
    case WQL3D_FO_TRUP: src = I.trup; nc = 1; break;
    default: return WQL3D_EINVAL;
  }
  if (cudaMemcpyAsync(out, src, sizeof(double) * nc * n, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return WQL3D_ECUDA;
  return WQL3D_OK;
}

}  // namespace wql3d
