// Kernels of the discrete adjoint of the elastic RK stage (see wql3d_adjoint.cuh).
#include "wql3d_adjoint.cuh"
#include "wql3d_stage.cuh"

namespace wql3d {

namespace {

// Pre-pass of reversed stage s at every point: R = DFbar + B_s dt Fbar (the
// rate adjoint of the stage), DFbar <- A_s R, the pointwise transposes Z and
// Y into ZY, and the material gradient from the forward derivative terms of
// the stage input Sprev (curv_derivs: the same conservative operator as the
// forward stage):
//   g_lambda += (R_xx + R_yy + R_zz) tr(grad v)
//   g_mu     += 2 (R_xx v_x,x + R_yy v_y,y + R_zz v_z,z) + R_xy (v_x,y + v_y,x) + ...
//   g_rho    += -1 / (rho^2 J) sum_f R_{v_f} (flux sum)_f
__global__ void __launch_bounds__(128, 3) k_adj_pre(Blk<double> b, AdjBlk A, double Bdt, double As,
                                                    const double *__restrict__ Sprev, const double *__restrict__ E) {
  int x, y, z;
  if (!flat_point(b, x, y, z)) return;
  const long long p = pidx(b, x, y, z);
  const long long V = b.vol;
  // R is kept in memory only where a later pass of the stage reads it: the
  // face points (k_adj_face) and the sources' support box (k_adj_moment)
  const bool keepR = x == 1 || x == b.nx || y == 1 || y == b.ny || z == 1 || z == b.nz ||
                     (x >= b.sbox[0] && x <= b.sbox[1] && y >= b.sbox[2] && y <= b.sbox[3] && z >= b.sbox[4] &&
                      z <= b.sbox[5]);
  double R[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    const double r = A.DFb[c * V + p] + Bdt * A.Fb[c * V + p];
    R[c] = r;
    if (keepR) A.R[c * V + p] = r;
    A.DFb[c * V + p] = As * r;
  }
  const double lam = b.M[p], mu = b.M[V + p], rho = b.M[2 * V + p];
  const double J = ld(b.J + p);
  const double a1 = 1.0 / (rho * J);
  const double l2m = lam + 2.0 * mu;
  // W_{r,f}: derivative of R_sigma . sigma_dot with respect to grad v (row r, component f)
  double W[3][3];
  W[0][0] = l2m * R[3] + lam * (R[4] + R[5]);
  W[1][1] = l2m * R[4] + lam * (R[3] + R[5]);
  W[2][2] = l2m * R[5] + lam * (R[3] + R[4]);
  W[0][1] = W[1][0] = mu * R[6];
  W[0][2] = W[2][0] = mu * R[7];
  W[1][2] = W[2][1] = mu * R[8];
  double *ZY = A.ZY + p;
#pragma unroll
  for (int f = 0; f < 3; ++f) ZY[f * V] = a1 * R[f];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double X0 = ld(b.met + (0 * 3 + a) * V + p), X1 = ld(b.met + (1 * 3 + a) * V + p);
    const double X2 = ld(b.met + (2 * 3 + a) * V + p);
#pragma unroll
    for (int f = 0; f < 3; ++f) ZY[(3 + a * 3 + f) * V] = X0 * W[0][f] + X1 * W[1][f] + X2 * W[2][f];
  }
  // derivative terms of the stage input: recorded by the forward pass, or
  // recomputed (e: normal and shear strain rates, fs: stress-flux sums)
  double e[6], fs[3];
  if (E) {
#pragma unroll
    for (int c = 0; c < 6; ++c) e[c] = E[c * V + p];
#pragma unroll
    for (int c = 0; c < 3; ++c) fs[c] = E[(6 + c) * V + p];
  } else {
    double U[9], S[9];
    curv_derivs<double>(b, Sprev, x, y, z, p, U, S);
    e[0] = U[0]; e[1] = U[4]; e[2] = U[8];
    e[3] = U[3] + U[1]; e[4] = U[6] + U[2]; e[5] = U[7] + U[5];
    fs[0] = S[0] + S[3] + S[6]; fs[1] = S[1] + S[4] + S[7]; fs[2] = S[2] + S[5] + S[8];
  }
  const double tr = e[0] + e[1] + e[2];
  double *g = A.g + p;
  g[0] += (R[3] + R[4] + R[5]) * tr;
  g[V] += 2.0 * (R[3] * e[0] + R[4] * e[1] + R[5] * e[2]) + R[6] * e[3] + R[7] * e[4] + R[8] * e[5];
  g[2 * V] += -a1 / rho * (R[0] * fs[0] + R[1] * fs[1] + R[2] * fs[2]);
}

// Gather pass: Fbar_v += sum_a (1/h_a) D_a^T Y_a, Fbar_sigma += J sum_a X_a (1/h_a) D_a^T Z
__global__ void __launch_bounds__(128, 4) k_adj_stencil(Blk<double> b, AdjBlk A) {
  int x, y, z;
  if (!flat_point(b, x, y, z)) return;
  const long long p = pidx(b, x, y, z);
  const long long V = b.vol;
  const int pos[3] = {x, y, z};
  const long long st[3] = {1, b.sy, b.sz};
  const double ih[3] = {b.ihq, b.ihr, b.ihs};
  double fv[3] = {0, 0, 0};
  double T[3][3];
#pragma unroll 1
  for (int a = 0; a < 3; ++a) {
    double ty[3] = {0, 0, 0}, tz[3] = {0, 0, 0};
    const int *to = A.toff[a] + (pos[a] - 1) * ADJ_TW;
    const double *tc = A.tc[a] + (pos[a] - 1) * ADJ_TW;
#pragma unroll
    for (int k = 0; k < ADJ_TW; ++k) {
      const double c = __ldg(tc + k);
      if (c == 0.0) continue;
      const long long q = p + (long long)__ldg(to + k) * st[a];
#pragma unroll
      for (int f = 0; f < 3; ++f) {
        tz[f] = tz[f] + c * ld(A.ZY + f * V + q);
        ty[f] = ty[f] + c * ld(A.ZY + (3 + a * 3 + f) * V + q);
      }
    }
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      fv[f] = fv[f] + ih[a] * ty[f];
      T[a][f] = ih[a] * tz[f];
    }
  }
  double P[3][3];  // P_{r,f} = sum_a X_{r,a} T_{a,f}
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const double X0 = ld(b.met + (r * 3 + 0) * V + p), X1 = ld(b.met + (r * 3 + 1) * V + p);
    const double X2 = ld(b.met + (r * 3 + 2) * V + p);
#pragma unroll
    for (int f = 0; f < 3; ++f) P[r][f] = X0 * T[0][f] + X1 * T[1][f] + X2 * T[2][f];
  }
  const double J = ld(b.J + p);
  double *Fb = A.Fb + p;
  Fb[0] += fv[0];
  Fb[V] += fv[1];
  Fb[2 * V] += fv[2];
  Fb[3 * V] += J * P[0][0];
  Fb[4 * V] += J * P[1][1];
  Fb[5 * V] += J * P[2][2];
  Fb[6 * V] += J * (P[1][0] + P[0][1]);
  Fb[7 * V] += J * (P[2][0] + P[0][2]);
  Fb[8 * V] += J * (P[2][1] + P[1][2]);
}

// Face pass: the SAT term DF(p) -= pen * structure(bc(u(p))) of every face
// point with a physical boundary condition, in the reference's face order:
// Fbar(p) -= Jac^T R(p) and the material gradient by dual numbers at the
// stage input.  Edge and corner points belong to several faces: atomics.
__global__ void __launch_bounds__(128) k_adj_face(Blk<double> b, AdjBlk A, const double *__restrict__ Sprev,
                                                 int f, int count) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const int axis = f >> 1, plus = f & 1;
  const int d0 = axis == 0 ? b.ny : b.nx;
  const int a1 = k / d0, a0 = k - a1 * d0;
  const int fixed = plus ? (axis == 0 ? b.nx : axis == 1 ? b.ny : b.nz) : 1;
  int x, y, z;
  if (axis == 0) { x = fixed; y = a0 + 1; z = a1 + 1; }
  else if (axis == 1) { x = a0 + 1; y = fixed; z = a1 + 1; }
  else { x = a0 + 1; y = a1 + 1; z = fixed; }
  const long long p = pidx(b, x, y, z);
  const long long V = b.vol;
  const int type = b.bc[f];
  const double r = type == 1 ? 0.0 : type == 2 ? 1.0 : -1.0;
  const double lam = b.M[p], mu = b.M[V + p], rho = b.M[2 * V + p];
  const double qx = ld(b.met + (long long)(0 + axis) * V + p);
  const double qy = ld(b.met + (long long)(3 + axis) * V + p);
  const double qz = ld(b.met + (long long)(6 + axis) * V + p);
  const double norm = sqrt(qx * qx + qy * qy + qz * qz);
  const double h = axis == 0 ? b.hq : axis == 1 ? b.hr : b.hs;
  const double pen = b.tau0 / h;
  double l[3], m[3], n[3];
  if (b.nrm[f]) {
    const long long fn = (long long)d0 * (axis == 2 ? b.ny : b.nz);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      l[c] = ld(b.nrm[f] + (0 + c) * fn + k);
      m[c] = ld(b.nrm[f] + (3 + c) * fn + k);
      n[c] = ld(b.nrm[f] + (6 + c) * fn + k);
    }
  } else {
    cart_basis<double>(axis, l, m, n);
  }
  double R[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) R[c] = A.R[c * V + p];
  // transposed Jacobian: column j of the (linear) SAT term
  for (int j = 0; j < 9; ++j) {
    double u[9], out[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) u[c] = c == j ? 1.0 : 0.0;
    sat_term<double>(plus, u, rho, mu, lam, l, m, n, norm, r, pen, out);
    double acc = 0.0;
#pragma unroll
    for (int c = 0; c < 9; ++c) acc += out[c] * R[c];
    atomicAdd(A.Fb + j * V + p, -acc);
  }
  // material derivatives at the stage input
  Dual u[9], ld3[3], md3[3], nd3[3];
#pragma unroll
  for (int c = 0; c < 9; ++c) u[c] = Dual(Sprev[c * V + p]);
#pragma unroll
  for (int c = 0; c < 3; ++c) { ld3[c] = Dual(l[c]); md3[c] = Dual(m[c]); nd3[c] = Dual(n[c]); }
  for (int prm = 0; prm < 3; ++prm) {
    const Dual dl(lam, prm == 0 ? 1.0 : 0.0), dm(mu, prm == 1 ? 1.0 : 0.0), dr(rho, prm == 2 ? 1.0 : 0.0);
    Dual out[9];
    sat_term<Dual>(plus, u, dr, dm, dl, ld3, md3, nd3, Dual(norm), Dual(r), Dual(pen), out);
    double acc = 0.0;
#pragma unroll
    for (int c = 0; c < 9; ++c) acc += out[c].b * R[c];
    atomicAdd(A.g + prm * V + p, -acc);
  }
}

// moment-tensor gradient of the sources at the stage time t: one block per
// source over its delta support, gM[6 i + c] -= A_i(t) sum delta R_(3+c)
__global__ void __launch_bounds__(256) k_adj_moment(Blk<double> b, AdjBlk A, double t) {
  const int i = blockIdx.x;
  const DevSource &s = b.src[i];
  __shared__ double red[6][256];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  if (s.near[0] >= 1) {
    const int hw = b.src_half, w = 2 * hw + 1;
    const double At = source_time(s.type, t, s.par[1], s.par[0]);
    for (int j = threadIdx.x; j < w * w * w; j += blockDim.x) {
      const int x = s.near[0] - hw + j % w, y = s.near[1] - hw + (j / w) % w, z = s.near[2] - hw + j / (w * w);
      if (x < 1 || x > b.nx || y < 1 || y > b.ny || z < 1 || z > b.nz) continue;
      const long long p = pidx(b, x, y, z);
      const double hx = b.hq / diag_metric<double, MESH_CURV>(b, 0, x, y, z, p);
      const double hy = b.hr / diag_metric<double, MESH_CURV>(b, 1, x, y, z, p);
      const double hz = b.hs / diag_metric<double, MESH_CURV>(b, 2, x, y, z, p);
      const double delta = singular_source(x, s.near[0], hx, (s.par[8] - s.phys[0]) / hx, b.src_order, b.src_alpha) *
                           singular_source(y, s.near[1], hy, (s.par[9] - s.phys[1]) / hy, b.src_order, b.src_alpha) *
                           singular_source(z, s.near[2], hz, (s.par[10] - s.phys[2]) / hz, b.src_order, b.src_alpha);
#pragma unroll
      for (int c = 0; c < 6; ++c) acc[c] -= At * delta * A.R[(3 + c) * b.vol + p];
    }
  }
#pragma unroll
  for (int c = 0; c < 6; ++c) red[c][threadIdx.x] = acc[c];
  __syncthreads();
  for (int sh = blockDim.x / 2; sh > 0; sh >>= 1) {
    if (threadIdx.x < sh)
#pragma unroll
      for (int c = 0; c < 6; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + sh];
    __syncthreads();
  }
  if (threadIdx.x < 6) A.gM[6 * i + threadIdx.x] += red[threadIdx.x][0];
}

// receiver residuals of one sample into the velocity adjoint at the stations' nodes
__global__ void k_adj_receivers(Blk<double> b, AdjBlk A) {
  for (int r = threadIdx.x; r < b.nrec; r += blockDim.x) {
    const int i = b.ridx[3 * r], j = b.ridx[3 * r + 1], k = b.ridx[3 * r + 2];
    if (i <= 0 || j <= 0 || k <= 0) continue;
    const long long p = pidx(b, i, j, k);
#pragma unroll
    for (int c = 0; c < 3; ++c) atomicAdd(A.Fb + c * b.vol + p, A.res[3 * r + c]);
  }
}

}  // namespace

void adj_launch_stage(const Blk<double> &b, const AdjBlk &A, int stage, double Bdt, double A_s, cudaStream_t s,
                      int64_t *launches) {
  const long long npts = (long long)b.nx * b.ny * b.nz;
  const unsigned gr = (unsigned)((npts + 127) / 128);
  k_adj_pre<<<gr, 128, 0, s>>>(b, A, Bdt, A_s, A.S[stage - 1], A.E[stage - 1]);
  ++*launches;
  for (int f = 0; f < 6; ++f) {
    if (b.bc[f] <= 0) continue;
    const int axis = f >> 1;
    const int count = axis == 0 ? b.ny * b.nz : axis == 1 ? b.nx * b.nz : b.nx * b.ny;
    k_adj_face<<<(count + 127) / 128, 128, 0, s>>>(b, A, A.S[stage - 1], f, count);
    ++*launches;
  }
  k_adj_stencil<<<gr, 128, 0, s>>>(b, A);
  ++*launches;
}

void adj_launch_moment(const Blk<double> &b, const AdjBlk &A, double t, cudaStream_t s, int64_t *launches) {
  if (b.nsrc <= 0) return;
  k_adj_moment<<<b.nsrc, 256, 0, s>>>(b, A, t);
  ++*launches;
}

void adj_launch_receivers(const Blk<double> &b, const AdjBlk &A, cudaStream_t s, int64_t *launches) {
  if (b.nrec <= 0) return;
  k_adj_receivers<<<1, 128, 0, s>>>(b, A);
  ++*launches;
}

int upload_tables_adjoint(const void *t) { return upload_tables_here(*(const ConstTables *)t); }

}  // namespace wql3d
