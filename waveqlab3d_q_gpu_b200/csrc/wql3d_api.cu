// C ABI of the B200-native WaveQLab3D per-step volume update (see include/wql3d.h).
//
// Host side: block setup (padded HBM layout, per-axis Cartesian metrics,
// device-computed curvilinear metrics, face bases, PML slabs, memory
// variables, source and receiver lookup), the RK stage sequence of
// src/time_step.f90:68-150, CUDA-graph capture of the step loop, and the
// host <-> device residency calls.
#include "wql3d.h"
#include "wql3d_device.cuh"
#include "wql3d_iface.cuh"
#include "wql3d_stage.cuh"
#include "wql3d_adjoint.cuh"
#include "wql3d_batch.cuh"
#include "wql3d_upwind.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

using namespace wql3d;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

#define CK(call)                                                                                  \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess)                                                                        \
      return fail(e_ == cudaErrorMemoryAllocation ? WQL3D_ENOMEM : WQL3D_ECUDA,                   \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                            \
  } while (0)

const double kRkA[5] = {0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
                        -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0};
const double kRkB[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                        1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                        2277821191437.0 / 14882151754819.0};
const double kRkC[6] = {0.0, 1432997174477.0 / 9575080441755.0, 2526269341429.0 / 6820363962896.0,
                        2006345519317.0 / 3224310063776.0, 2802321613138.0 / 2924317926251.0, 1.0};

// SBP rows 1..6 of the traditional-6 first-derivative operator, in the
// reference's summation order (src/JU_xJU_yJU_z6.f90:74-161, src/metrics.f90:29-86)
const int kSbpCnt[6] = {6, 5, 5, 6, 7, 8};
const int kSbpIdx[6][8] = {{6, 5, 4, 3, 2, 1, 0, 0}, {6, 5, 4, 3, 1, 0, 0, 0}, {6, 5, 4, 2, 1, 0, 0, 0},
                           {7, 6, 5, 3, 2, 1, 0, 0}, {8, 7, 6, 4, 3, 2, 1, 0}, {9, 8, 7, 5, 4, 3, 2, 1}};
double kSbpC[2][6][8];

void sbp_tables() {
  static bool done = false;
  if (done) return;
  const double rows[6][8] = {
      {0.036577936277544, 0.104488069284042, -0.450398306578272, -0.141512858744873, 2.033378678700676, -1.582533518939116, 0, 0},
      {-0.014903449191300, -0.069112065532624, 0.258816087376832, 0.287258622978251, -0.462059195631158, 0, 0, 0},
      {-0.018129342917256, -0.022902190275815, 0.606235523609147, -0.636451095137907, 0.071247104721830, 0, 0, 0},
      {0.013435342414630, -0.051642265516119, 0.520262285050482, -0.306681191361148, -0.290087484386815, 0.114713313798970, 0, 0},
      {0.018281071473911, -0.164529643265203, 0.769199413962647, -0.707905442575989, 0.015764336127392, 0.105400944933782, -0.036210680656541, 0},
      {0.016437980868017, -0.147941827812150, 0.739709139060752, -0.691649024426814, 0.063183694641876, 0.011220896474665, 0.020437334208704, -0.011398193015050}};
  for (int lit = 0; lit < 2; ++lit)
    for (int r = 0; r < 6; ++r)
      for (int k = 0; k < 8; ++k) kSbpC[lit][r][k] = rows[r][k];
  // row 4 coefficient of point 7 as a single-precision literal
  kSbpC[1][3][0] = (double)0.013435342414630f;
  done = true;
}

// host copy of the SBP stencil at 1-based i of an axis of n points
void host_row(int i, int n, int lit, int &cnt, int idx[8], double c[8]) {
  if (i >= 7 && i <= n - 6) {
    const double cc[6] = {-1.0 / 60.0, 0.15, -0.75, 0.75, -0.15, 1.0 / 60.0};
    const int off[6] = {-3, -2, -1, 1, 2, 3};
    cnt = 6;
    for (int k = 0; k < 6; ++k) { idx[k] = i + off[k]; c[k] = cc[k]; }
    return;
  }
  if (i >= n - 5) {
    int r = n - i;
    cnt = kSbpCnt[r];
    for (int k = 0; k < cnt; ++k) { idx[k] = n + 1 - kSbpIdx[r][k]; c[k] = -kSbpC[lit][r][k]; }
    return;
  }
  int r = i - 1;
  cnt = kSbpCnt[r];
  for (int k = 0; k < cnt; ++k) { idx[k] = kSbpIdx[r][k]; c[k] = kSbpC[lit][r][k]; }
}

struct Alloc {
  std::vector<void *> ptrs;
  int64_t bytes = 0;
  cudaStream_t stream = nullptr;  // zero-fills are ordered on the owning domain's stream
  template <typename P>
  cudaError_t get(P **p, size_t n, bool zero = true) {
    void *v = nullptr;
    size_t nb = n * sizeof(P);
    if (nb == 0) nb = 16;
    cudaError_t e = cudaMalloc(&v, nb);
    if (e != cudaSuccess) return e;
    if (zero) {
      e = cudaMemsetAsync(v, 0, nb, stream);
      if (e != cudaSuccess) {
        cudaFree(v);
        return e;
      }
    }
    ptrs.push_back(v);
    bytes += (int64_t)nb;
    *p = (P *)v;
    return cudaSuccess;
  }
  void release() {
    for (void *p : ptrs) cudaFree(p);
    ptrs.clear();
  }
};

}  // namespace

namespace wql3d {
// lets other translation units of the library set the wql3d_last_error() text
void set_last_error(const std::string &msg) { g_err = msg; }
}  // namespace wql3d

struct HostBlock {
  int nq = 0, nr = 0, ns = 0;
  int mesh = 0;
  int PX = 0, PY = 0, PZ = 0;   // padded extents
  int XOFF = 4;
  long long vol = 0;
  std::vector<double> coords;   // 3 * nq*nr*ns (host copy for source / receiver lookup)
  std::vector<int> ridx;
  int nrec = 0;
  int nsrc = 0;
  int iface_side[2] = {0, 0};
};

struct wql3d_domain {
  wql3d_domain_desc desc;
  int nblocks = 0;
  int fp32 = 0;
  int response = 0;
  int nmech = 0;
  cudaStream_t stream = nullptr;
  // second stream for the Cartesian near-boundary shell, forked from and
  // joined back to `stream` every stage (the shell overlaps the interior)
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  Alloc mem;
  HostBlock hb[2];
  Blk<double> bd[2];
  Blk<float> bf[2];
  int cur = 0;
  DevTime *time = nullptr;
  // interface
  bool has_iface = false;
  IfaceDev iface;
  // graph cache
  cudaGraphExec_t graph = nullptr;
  double g_dt = 0.0;
  int g_w = -1, g_cur = -1;
  int64_t g_launches = 0;         // kernels in one replay of the captured two-step graph
  int64_t launches = 0;
  double *red = nullptr;
  int *flag = nullptr;
  // s-slab ghost-plane exchange buffers (2 faces x up to 10 x 3 x nr x nq)
  bool slab = false;
  void *halo_send = nullptr, *halo_recv = nullptr;
  // discrete adjoint (wql3d_adjoint_enable)
  bool adj_on = false;
  AdjBlk adj;
  double *adj_res = nullptr;   // receiver residuals of one sample (device)
  // plane extraction (wql3d_get_plane): largest plane x 9 components
  double *plane = nullptr;
  long long plane_cap = 0;
  // host <-> device staging: 9 components of the largest block with 3 ghost layers
  double *xfer = nullptr;
  long long xfer_cap = 0;
};

namespace {

template <typename T>
Blk<T> &blk(wql3d_domain *d, int i);
template <>
Blk<double> &blk<double>(wql3d_domain *d, int i) { return d->bd[i]; }
template <>
Blk<float> &blk<float>(wql3d_domain *d, int i) { return d->bf[i]; }

int upload_constants() {
  sbp_tables();
  int cnt[6], idx[6][8];
  for (int r = 0; r < 6; ++r) {
    cnt[r] = kSbpCnt[r];
    for (int k = 0; k < 8; ++k) idx[r][k] = kSbpIdx[r][k];
  }
  CK(cudaMemcpyToSymbol(c_sbp_cnt, cnt, sizeof(cnt)));
  CK(cudaMemcpyToSymbol(c_sbp_idx, idx, sizeof(idx)));
  // c_sbp_c[0] = double literal, [1] = single literal
  CK(cudaMemcpyToSymbol(c_sbp_c, kSbpC, sizeof(kSbpC)));
  CK(cudaMemcpyToSymbol(c_rkA, kRkA, sizeof(kRkA)));
  CK(cudaMemcpyToSymbol(c_rkB, kRkB, sizeof(kRkB)));
  CK(cudaMemcpyToSymbol(c_rkC, kRkC, sizeof(kRkC)));
  // the same tables into each stage-launcher translation unit's constants
  ConstTables t;
  memcpy(t.sbp_cnt, cnt, sizeof(cnt));
  memcpy(t.sbp_idx, idx, sizeof(idx));
  memcpy(t.sbp_c, kSbpC, sizeof(kSbpC));
  memcpy(t.rkA, kRkA, sizeof(kRkA));
  memcpy(t.rkB, kRkB, sizeof(kRkB));
  memcpy(t.rkC, kRkC, sizeof(kRkC));
  int (*const up[])(const ConstTables &) = {upload_tables_cart_f64,    upload_tables_cart_f32,
                                            upload_tables_curv_f64,    upload_tables_curv_f32,
                                            upload_tables_generic_f64, upload_tables_generic_f32,
                                            upload_tables_batch_f64,   upload_tables_batch_f32};
  for (auto f : up) {
    const int e = f(t);
    if (e != 0) return fail(WQL3D_ECUDA, std::string("stage constants: ") + cudaGetErrorString((cudaError_t)e));
  }
  if (const int e = upload_tables_adjoint(&t))
    return fail(WQL3D_ECUDA, std::string("adjoint constants: ") + cudaGetErrorString((cudaError_t)e));
  return WQL3D_OK;
}

// copy one padded device component <-> host component with ghost width hnb
int copy_component(wql3d_domain *d, const HostBlock &h, void *dev, size_t esz, void *host, int hnb, bool to_dev) {
  cudaMemcpy3DParms p;
  memset(&p, 0, sizeof(p));
  cudaPitchedPtr hp = make_cudaPitchedPtr(host, (size_t)(h.nq + 2 * hnb) * esz, h.nq + 2 * hnb, h.nr + 2 * hnb);
  cudaPitchedPtr dp = make_cudaPitchedPtr(dev, (size_t)h.PX * esz, h.PX, h.PY);
  cudaPos hpos = make_cudaPos((size_t)hnb * esz, hnb, hnb);
  cudaPos dpos = make_cudaPos((size_t)h.XOFF * esz, NB, NB);
  if (to_dev) { p.srcPtr = hp; p.srcPos = hpos; p.dstPtr = dp; p.dstPos = dpos; p.kind = cudaMemcpyHostToDevice; }
  else { p.srcPtr = dp; p.srcPos = dpos; p.dstPtr = hp; p.dstPos = hpos; p.kind = cudaMemcpyDeviceToHost; }
  p.extent = make_cudaExtent((size_t)h.nq * esz, h.nr, h.ns);
  CK(cudaMemcpy3DAsync(&p, d->stream));
  return WQL3D_OK;
}

// Host arrays move through a contiguous device staging buffer: one copy of
// up to 9 components at the link's full rate, then a kernel that scatters
// them into (or gathers them from) the padded device layout, converting to
// the storage precision on the device.  (A 3-D strided copy moves one host
// row, a few hundred bytes, per DMA transfer.)
struct XferGeom {
  int nq, nr, ns, hnb;          // interior extents and the host array's ghost width
  long long PX, PY, XOFF, NBZ;  // padded device layout: x pitch, y pitch, x / y-z offsets
  long long vol;                // device component stride
};

template <typename T>
__global__ void k_xfer(XferGeom g, double *stage, T *dev, int nc, int to_dev) {
  const long long hq = g.nq + 2 * g.hnb, hr = g.nr + 2 * g.hnb, hs = g.ns + 2 * g.hnb;
  const long long hn = hq * hr * hs;
  const long long n = (long long)g.nq * g.nr * g.ns;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n * nc;
       i += (long long)gridDim.x * blockDim.x) {
    const long long c = i / n, k = i - c * n;
    const long long x = k % g.nq, y = (k / g.nq) % g.nr, z = k / ((long long)g.nq * g.nr);
    const long long hi = c * hn + (x + g.hnb) + hq * ((y + g.hnb) + hr * (z + g.hnb));
    const long long di = c * g.vol + (g.XOFF + x) + g.PX * ((g.NBZ + y) + g.PY * (g.NBZ + z));
    if (to_dev) dev[di] = (T)stage[hi];
    else stage[hi] = (double)dev[di];
  }
}

template <typename T>
int xfer_array(wql3d_domain *d, const HostBlock &h, T *dev, int ncomp, double *host, int hnb, bool to_dev) {
  const long long hn = (long long)(h.nq + 2 * hnb) * (h.nr + 2 * hnb) * (h.ns + 2 * hnb);
  XferGeom g{h.nq, h.nr, h.ns, hnb, h.PX, h.PY, h.XOFF, NB, h.vol};
  for (int c0 = 0; c0 < ncomp; c0 += 9) {
    const int nc = std::min(9, ncomp - c0);
    const size_t bytes = sizeof(double) * (size_t)(hn * nc);
    double *hp = host + (long long)c0 * hn;
    const long long n = (long long)h.nq * h.nr * h.ns * nc;
    const unsigned gr = (unsigned)std::min<long long>((n + 255) / 256, 148LL * 32);
    if (to_dev) {
      CK(cudaMemcpyAsync(d->xfer, hp, bytes, cudaMemcpyHostToDevice, d->stream));
      k_xfer<T><<<gr, 256, 0, d->stream>>>(g, d->xfer, dev + (long long)c0 * h.vol, nc, 1);
    } else {
      if (hnb > 0) CK(cudaMemsetAsync(d->xfer, 0, bytes, d->stream));
      k_xfer<T><<<gr, 256, 0, d->stream>>>(g, d->xfer, const_cast<T *>(dev) + (long long)c0 * h.vol, nc, 0);
      CK(cudaMemcpyAsync(hp, d->xfer, bytes, cudaMemcpyDeviceToHost, d->stream));
    }
    CK(cudaGetLastError());
    // the staging buffer is reused by the next chunk and the host data must
    // be complete (or consumed) on return
    CK(cudaStreamSynchronize(d->stream));
  }
  return WQL3D_OK;
}

// double host data -> device storage type (FP32 path converts on the host)
template <typename T>
int put_array(wql3d_domain *d, const HostBlock &h, T *dev, int ncomp, const double *host, int hnb) {
  long long hn = (long long)(h.nq + 2 * hnb) * (h.nr + 2 * hnb) * (h.ns + 2 * hnb);
  if (d->xfer && hn * 9 <= d->xfer_cap) return xfer_array<T>(d, h, dev, ncomp, const_cast<double *>(host), hnb, true);
  for (int c = 0; c < ncomp; ++c) {
    const double *src = host + (long long)c * hn;
    if (sizeof(T) == sizeof(double)) {
      int rc = copy_component(d, h, (void *)(dev + (long long)c * h.vol), sizeof(double), (void *)src, hnb, true);
      if (rc) return rc;
    } else {
      std::vector<T> tmp((size_t)hn);
      for (long long i = 0; i < hn; ++i) tmp[(size_t)i] = (T)src[i];
      int rc = copy_component(d, h, (void *)(dev + (long long)c * h.vol), sizeof(T), tmp.data(), hnb, true);
      if (rc) return rc;
      CK(cudaStreamSynchronize(d->stream));
    }
  }
  return WQL3D_OK;
}

template <typename T>
int get_array(wql3d_domain *d, const HostBlock &h, const T *dev, int ncomp, double *host, int hnb) {
  long long hn = (long long)(h.nq + 2 * hnb) * (h.nr + 2 * hnb) * (h.ns + 2 * hnb);
  if (d->xfer && hn * 9 <= d->xfer_cap) return xfer_array<T>(d, h, const_cast<T *>(dev), ncomp, host, hnb, false);
  for (int c = 0; c < ncomp; ++c) {
    double *dst = host + (long long)c * hn;
    if (sizeof(T) == sizeof(double)) {
      int rc = copy_component(d, h, (void *)(dev + (long long)c * h.vol), sizeof(double), (void *)dst, hnb, false);
      if (rc) return rc;
    } else {
      std::vector<T> tmp((size_t)hn, (T)0);
      int rc = copy_component(d, h, (void *)(dev + (long long)c * h.vol), sizeof(T), tmp.data(), hnb, false);
      if (rc) return rc;
      CK(cudaStreamSynchronize(d->stream));
      for (long long i = 0; i < hn; ++i) dst[i] = (double)tmp[(size_t)i];
    }
  }
  CK(cudaStreamSynchronize(d->stream));
  return WQL3D_OK;
}

// curvilinear metrics from coordinates: src/grid.f90:398-471 with the SBP
// operator of src/metrics.f90:16-491 (setup-time kernel)
template <typename T>
__global__ void k_metrics(Blk<T> b, const double *X, double *met, double *Jout) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int r = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int s = blockIdx.z * blockDim.z + threadIdx.z + 1;
  if (q > b.nx || r > b.ny || s > b.nz) return;
  const long long p = pidx(b, q, r, s);
  const long long V = b.vol;
  const int pos[3] = {q, r, s};
  const int nn[3] = {b.nx, b.ny, b.nz};
  const long long st[3] = {1, b.sy, b.sz};
  const int ng[3] = {b.nx, b.ny, b.nzg};
  double D[3][3];  // D[axis][comp]
  for (int a = 0; a < 3; ++a) {
    Row row;
    sbp_row(pos[a], nn[a], b.lit, row, b.open_lo[a], b.open_hi[a]);
    double h = 1.0 / (double)(ng[a] - 1);
    for (int c = 0; c < 3; ++c) {
      double sum = 0.0;
      for (int k = 0; k < row.cnt; ++k) sum = __dadd_rn(sum, __dmul_rn(row.c[k], X[c * V + p + row.off[k] * st[a]]));
      D[a][c] = __dmul_rn(1.0 / h, sum);
    }
  }
  const double *Xq = D[0], *Xr = D[1], *Xs = D[2];
  double J = __dadd_rn(__dsub_rn(__dmul_rn(Xq[0], __dsub_rn(__dmul_rn(Xr[1], Xs[2]), __dmul_rn(Xr[2], Xs[1]))),
                                 __dmul_rn(Xq[1], __dsub_rn(__dmul_rn(Xr[0], Xs[2]), __dmul_rn(Xr[2], Xs[0])))),
                       __dmul_rn(Xq[2], __dsub_rn(__dmul_rn(Xr[0], Xs[1]), __dmul_rn(Xr[1], Xs[0]))));
  double iJ = 1.0 / J;
  double m[9];
  m[0] = __dmul_rn(iJ, __dsub_rn(__dmul_rn(Xr[1], Xs[2]), __dmul_rn(Xr[2], Xs[1])));
  m[1] = __dmul_rn(iJ, __dsub_rn(__dmul_rn(Xq[2], Xs[1]), __dmul_rn(Xq[1], Xs[2])));
  m[2] = __dmul_rn(iJ, __dsub_rn(__dmul_rn(Xq[1], Xr[2]), __dmul_rn(Xq[2], Xr[1])));
  m[3] = __dmul_rn(iJ, __dsub_rn(__dmul_rn(Xr[2], Xs[0]), __dmul_rn(Xr[0], Xs[2])));
  m[4] = __dmul_rn(iJ, __dsub_rn(__dmul_rn(Xq[0], Xs[2]), __dmul_rn(Xq[2], Xs[0])));
  m[5] = __dmul_rn(iJ, __dsub_rn(__dmul_rn(Xq[2], Xr[0]), __dmul_rn(Xq[0], Xr[2])));
  m[6] = __dmul_rn(iJ, __dsub_rn(__dmul_rn(Xr[0], Xs[1]), __dmul_rn(Xr[1], Xs[0])));
  m[7] = __dmul_rn(iJ, __dsub_rn(__dmul_rn(Xq[1], Xs[0]), __dmul_rn(Xq[0], Xs[1])));
  m[8] = __dmul_rn(iJ, __dsub_rn(__dmul_rn(Xq[0], Xr[1]), __dmul_rn(Xq[1], Xr[0])));
  for (int k = 0; k < 9; ++k) met[k * V + p] = m[k];
  Jout[p] = J;
}

// one field component set to v at every point of a block (init_vel_state)
template <typename T>
__global__ void k_fill_component(Blk<T> b, T *F, int c, T v) {
  int x, y, z;
  if (!flat_point(b, x, y, z)) return;
  F[(long long)c * b.vol + pidx(b, x, y, z)] = v;
}

// Components c0 .. c0 + nc - 1 of the fields on the plane of 1-based index
// `index` normal to axis dir (0: q, 1: r, 2: s) into a dense buffer: the
// first in-plane index (q, or r for dir 0) fastest, then the second, then
// the component (the extract_local_plane / write_slice layouts of
// src/plane_output.f90:594-653 and src/slice_output.f90:79-94).
template <typename T>
__global__ void k_plane_gather(Blk<T> b, const T *F, int dir, int index, int c0, int nc, double *out) {
  const int n1 = dir == 0 ? b.ny : b.nx, n2 = dir == 2 ? b.ny : b.nz;
  const long long total = (long long)n1 * n2 * nc;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int i1 = (int)(i % n1), i2 = (int)((i / n1) % n2), c = (int)(i / ((long long)n1 * n2));
    int x, y, z;
    if (dir == 0) { x = index; y = i1 + 1; z = i2 + 1; }
    else if (dir == 1) { x = i1 + 1; y = index; z = i2 + 1; }
    else { x = i1 + 1; y = i2 + 1; z = index; }
    out[i] = (double)F[(long long)(c0 + c) * b.vol + pidx(b, x, y, z)];
  }
}

// Strict-interior rates of a Cartesian elastic traditional-6 block on the
// caller's arrays (cartesian_elastic_o6_interior_kernel of
// src/traditional_cartesian_rhs_openacc.f90): field, rate, metricx/y/z and
// material dimensioned (n1, n2, n3, .) as the caller holds them, the box
// [lo, lo + ext) in their 1-based indices.  Every product and sum in the
// reference's order without contraction, so the rates equal a plain IEEE
// evaluation of the same expressions.
struct CartRhsArgs {
  const double *field, *mx, *my, *mz, *mat;
  double *rate;
  int n1, n2, n3;
  int lo[3], ext[3];
  double cx[3], cy[3], cz[3];
};

__global__ void __launch_bounds__(256) k_trad_cart_rhs(CartRhsArgs a) {
  const long long vol = (long long)a.n1 * a.n2 * a.n3;
  const long long sy = a.n1, sz = (long long)a.n1 * a.n2;
  const long long npts = (long long)a.ext[0] * a.ext[1] * a.ext[2];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < npts;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = a.lo[0] + (int)(i % a.ext[0]);
    const int y = a.lo[1] + (int)((i / a.ext[0]) % a.ext[1]);
    const int z = a.lo[2] + (int)(i / ((long long)a.ext[0] * a.ext[1]));
    const long long p = (long long)(x - 1) + sy * (y - 1) + sz * (z - 1);
    const double mx = a.mx[p], my = a.my[vol + p], mz = a.mz[2 * vol + p];
    double dfx[9], dfy[9], dfz[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) { dfx[c] = 0.0; dfy[c] = 0.0; dfz[c] = 0.0; }
#pragma unroll
    for (int s = 1; s <= 3; ++s) {
      const double kx = __dmul_rn(mx, a.cx[s - 1]), ky = __dmul_rn(my, a.cy[s - 1]), kz = __dmul_rn(mz, a.cz[s - 1]);
#pragma unroll
      for (int c = 0; c < 9; ++c) {
        const double *f = a.field + c * vol + p;
        dfx[c] = __dadd_rn(dfx[c], __dmul_rn(kx, __dsub_rn(__ldg(f + s), __ldg(f - s))));
        dfy[c] = __dadd_rn(dfy[c], __dmul_rn(ky, __dsub_rn(__ldg(f + s * sy), __ldg(f - s * sy))));
        dfz[c] = __dadd_rn(dfz[c], __dmul_rn(kz, __dsub_rn(__ldg(f + s * sz), __ldg(f - s * sz))));
      }
    }
    const double lam = a.mat[p], mu = a.mat[vol + p];
    const double a1 = 1.0 / a.mat[2 * vol + p];
    const double a2 = __dadd_rn(lam, __dmul_rn(2.0, mu)), a3 = lam, a4 = mu;
    double *r = a.rate + p;
    r[0] = __dadd_rn(r[0], __dmul_rn(a1, __dadd_rn(__dadd_rn(dfx[3], dfy[6]), dfz[7])));
    r[vol] = __dadd_rn(r[vol], __dmul_rn(a1, __dadd_rn(__dadd_rn(dfx[6], dfy[4]), dfz[8])));
    r[2 * vol] = __dadd_rn(r[2 * vol], __dmul_rn(a1, __dadd_rn(__dadd_rn(dfx[7], dfy[8]), dfz[5])));
    r[3 * vol] = __dadd_rn(__dadd_rn(r[3 * vol], __dmul_rn(a2, dfx[0])), __dmul_rn(a3, __dadd_rn(dfy[1], dfz[2])));
    r[4 * vol] = __dadd_rn(__dadd_rn(r[4 * vol], __dmul_rn(a2, dfy[1])), __dmul_rn(a3, __dadd_rn(dfx[0], dfz[2])));
    r[5 * vol] = __dadd_rn(__dadd_rn(r[5 * vol], __dmul_rn(a2, dfz[2])), __dmul_rn(a3, __dadd_rn(dfx[0], dfy[1])));
    r[6 * vol] = __dadd_rn(r[6 * vol], __dmul_rn(a4, __dadd_rn(dfy[0], dfx[1])));
    r[7 * vol] = __dadd_rn(r[7 * vol], __dmul_rn(a4, __dadd_rn(dfz[0], dfx[2])));
    r[8 * vol] = __dadd_rn(r[8 * vol], __dmul_rn(a4, __dadd_rn(dfz[1], dfy[2])));
  }
}

template <typename T>
__global__ void k_convert(const double *src, T *dst, long long n) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long s = (long long)gridDim.x * blockDim.x;
  for (; i < n; i += s) dst[i] = (T)src[i];
}

// unit_normals.f90 face bases from the metric of the face (host)
void gen_orth(double l[3], double m[3], const double n[3]) {
  const double tol = 1.0e-12;
  m[0] = 0.0; m[1] = 1.0; m[2] = 0.0;
  double d1 = sqrt((n[0] - m[0]) * (n[0] - m[0]) + (n[1] - m[1]) * (n[1] - m[1]) + (n[2] - m[2]) * (n[2] - m[2]));
  double d2 = sqrt((n[0] + m[0]) * (n[0] + m[0]) + (n[1] + m[1]) * (n[1] + m[1]) + (n[2] + m[2]) * (n[2] + m[2]));
  if (!(d1 >= tol && d2 >= tol)) { m[0] = 0.0; m[1] = 0.0; m[2] = 1.0; }
  double a = n[0] * m[0] + n[1] * m[1] + n[2] * m[2];
  for (int i = 0; i < 3; ++i) m[i] = m[i] - a * n[i];
  double s = 1.0 / sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
  for (int i = 0; i < 3; ++i) m[i] = s * m[i];
  l[0] = n[1] * m[2] - n[2] * m[1];
  l[1] = n[2] * m[0] - n[0] * m[2];
  l[2] = n[0] * m[1] - n[1] * m[0];
}

void nearest_moment(const HostBlock &h, double x1, double y1, double z1, int out[3]) {
  long long n1 = (long long)h.nq * h.nr * h.ns;
  const double *X = h.coords.data();
  double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
  for (long long i = 0; i < n1; ++i)
    for (int c = 0; c < 3; ++c) {
      double v = X[c * n1 + i];
      if (v < mn[c]) mn[c] = v;
      if (v > mx[c]) mx[c] = v;
    }
  double scale = 1.0;
  for (int c = 0; c < 3; ++c) scale = fmax(scale, fmax(fabs(mn[c]), fabs(mx[c])));
  double tol = 1000.0 * 2.220446049250313e-16 * scale;
  out[0] = out[1] = out[2] = -9999;
  if (!((mn[0] - tol <= x1 && x1 <= mx[0] + tol) && (mn[1] - tol <= y1 && y1 <= mx[1] + tol) &&
        (mn[2] - tol <= z1 && z1 <= mx[2] + tol)))
    return;
  double best = 1.0e8;
  for (int z = 1; z <= h.ns; ++z)
    for (int y = 1; y <= h.nr; ++y)
      for (int x = 1; x <= h.nq; ++x) {
        long long i = (x - 1) + (long long)h.nq * ((y - 1) + (long long)h.nr * (z - 1));
        double a = X[i] - x1, b = X[n1 + i] - y1, c = X[2 * n1 + i] - z1;
        double dist = sqrt(a * a + b * b + c * c);
        if (dist <= best) { out[0] = x; out[1] = y; out[2] = z; best = dist; }
      }
}

// Find_Coordinates, src/seismogram.f90:767-876
void nearest_receiver(const HostBlock &h, double x1, double y1, double z1, int out[3]) {
  long long n1 = (long long)h.nq * h.nr * h.ns;
  const double *X = h.coords.data();
  auto at = [&](int c, int x, int y, int z) { return X[c * n1 + (x - 1) + (long long)h.nq * ((y - 1) + (long long)h.nr * (z - 1))]; };
  out[0] = out[1] = out[2] = -9999;
  double best = 1.0e8;
  int px = h.nq, py = h.nr, pz = h.ns;
  for (int k = 1; k <= pz; ++k)
    for (int j = 1; j <= py; ++j)
      for (int i = 1; i <= px; ++i) {
        double hx = at(0, px, j, k) - at(0, px - 1, j, k);
        double hy = at(1, i, py, k) - at(1, i, py - 1, k);
        double hz = at(2, i, j, pz) - at(2, i, j, pz - 1);
        if (i < px) hx = at(0, i + 1, j, k) - at(0, i, j, k);
        if (j < py) hy = at(1, i, j + 1, k) - at(1, i, j, k);
        if (k < pz) hz = at(2, i, j, k + 1) - at(2, i, j, k);
        double a = at(0, i, j, k) - x1, b = at(1, i, j, k) - y1, c = at(2, i, j, k) - z1;
        double dist = sqrt(a * a + b * b + c * c);
        double dist0 = sqrt(hx * hx + hy * hy + hz * hz);
        if (dist <= best && dist <= 0.5 * dist0) { out[0] = i; out[1] = j; out[2] = k; best = dist; }
      }
}

template <typename T>
int setup_block(wql3d_domain *d, int bi) {
  const wql3d_block_desc &bd = d->desc.block[bi];
  HostBlock &h = d->hb[bi];
  Blk<T> &b = blk<T>(d, bi);
  memset(&b, 0, sizeof(b));
  if (bd.nq < 13 || bd.nr < 13 || bd.ns < 13) return fail(WQL3D_EINVAL, "each axis needs at least 13 points for the traditional-6 operator");
  if (bd.mesh != WQL3D_MESH_CARTESIAN && bd.mesh != WQL3D_MESH_CURVILINEAR) return fail(WQL3D_EINVAL, "unknown mesh kind");
  if (bd.mesh == WQL3D_MESH_CURVILINEAR && !bd.coords) return fail(WQL3D_EINVAL, "curvilinear block needs coordinates");
  if (!bd.material) return fail(WQL3D_EINVAL, "block material (lambda, mu, rho) is required");
  h.nq = bd.nq; h.nr = bd.nr; h.ns = bd.ns;
  h.mesh = bd.mesh;
  const int esz = (int)sizeof(T);
  h.XOFF = 32 / esz;  // first interior point of a row on a 32-byte boundary
  int row_elems = 128 / esz;
  h.PX = ((h.XOFF + h.nq + NB + row_elems - 1) / row_elems) * row_elems;
  h.PY = h.nr + 2 * NB;
  h.PZ = h.ns + 2 * NB;
  long long vol = (long long)h.PX * h.PY * h.PZ;
  vol = (vol + 63) / 64 * 64;
  h.vol = vol;
  b.nx = h.nq; b.ny = h.nr; b.nz = h.ns;
  b.sy = h.PX;
  b.sz = (long long)h.PX * h.PY;
  b.o1 = h.XOFF + b.sy * NB + b.sz * NB;
  b.vol = vol;
  b.lit = bd.f32_literal ? 1 : 0;
  // an s-slab of a larger block: global plane offset z0, nsg planes in all
  const bool slab = d->slab;
  const int z0 = slab ? d->desc.slab_z0 : 0;
  const int nsg = slab ? d->desc.slab_ns_global : h.ns;
  b.open_lo[2] = slab && z0 > 0 ? 1 : 0;
  b.open_hi[2] = slab && z0 + h.ns < nsg ? 1 : 0;
  b.nzg = nsg;
  b.hq = (T)(1.0 / (double)(h.nq - 1));
  b.hr = (T)(1.0 / (double)(h.nr - 1));
  b.hs = (T)(1.0 / (double)(nsg - 1));
  b.ihq = (T)(1.0 / (1.0 / (double)(h.nq - 1)));
  b.ihr = (T)(1.0 / (1.0 / (double)(h.nr - 1)));
  b.ihs = (T)(1.0 / (1.0 / (double)(nsg - 1)));
  const double cc[3] = {0.75, -0.15, 1.0 / 60.0};
  for (int s = 0; s < 3; ++s) {
    b.cx[s] = (T)(cc[s] / (1.0 / (double)(h.nq - 1)));
    b.cy[s] = (T)(cc[s] / (1.0 / (double)(h.nr - 1)));
    b.cz[s] = (T)(cc[s] / (1.0 / (double)(nsg - 1)));
  }
  b.tau0 = (T)bd.tau0;
  for (int f = 0; f < 6; ++f) b.bc[f] = bd.bc[f];
  {
    // closure rows 1..6 and their right mirrors as (offset, coefficient),
    // zero-padded to 8 taps, in the reference's summation order
    std::vector<double> rc(12 * 8, 0.0);
    std::vector<int> ro(12 * 8, 0);
    for (int r = 0; r < 6; ++r)
      for (int k = 0; k < kSbpCnt[r]; ++k) {
        rc[r * 8 + k] = kSbpC[b.lit][r][k];
        ro[r * 8 + k] = kSbpIdx[r][k] - (r + 1);
        rc[(6 + r) * 8 + k] = -kSbpC[b.lit][r][k];
        ro[(6 + r) * 8 + k] = (r + 1) - kSbpIdx[r][k];
      }
    double *drc;
    int *dro;
    CK(d->mem.get(&drc, rc.size()));
    CK(d->mem.get(&dro, ro.size()));
    CK(cudaMemcpyAsync(drc, rc.data(), sizeof(double) * rc.size(), cudaMemcpyHostToDevice, d->stream));
    CK(cudaMemcpyAsync(dro, ro.data(), sizeof(int) * ro.size(), cudaMemcpyHostToDevice, d->stream));
    CK(cudaStreamSynchronize(d->stream));
    b.rowc = drc;
    b.rowo = dro;
  }
  b.fd = bd.fd_operator;
  if (const UpwindTable *up = upwind_table(b.fd)) {
    // device rows of the upwind pair: D+ left, D+ right, D- left, D- right
    // (w rows each), then the near-boundary routine's D+ and D- interior
    // rows; offsets relative to the point, kUpSlots slots per row.  The right
    // rows of each operator are the negated mirror of the other's left rows.
    const int w = up->width, nrow = 4 * w + 2;
    std::vector<double> rc((size_t)nrow * kUpSlots, 0.0);
    std::vector<int> ro((size_t)nrow * kUpSlots, 0), rn((size_t)nrow, 0);
    for (int r = 0; r < w; ++r) {
      rn[r] = rn[3 * w + r] = up->pcnt[r];
      for (int k = 0; k < up->pcnt[r]; ++k) {
        rc[(size_t)r * kUpSlots + k] = up->pc[r][k];                    // D+ left
        ro[(size_t)r * kUpSlots + k] = up->pidx[r][k] - (r + 1);
        rc[(size_t)(3 * w + r) * kUpSlots + k] = -up->pc[r][k];         // D- right (mirror of D+ left)
        ro[(size_t)(3 * w + r) * kUpSlots + k] = (r + 1) - up->pidx[r][k];
      }
      rn[2 * w + r] = rn[w + r] = up->mcnt[r];
      for (int k = 0; k < up->mcnt[r]; ++k) {
        rc[(size_t)(2 * w + r) * kUpSlots + k] = up->mc[r][k];          // D- left
        ro[(size_t)(2 * w + r) * kUpSlots + k] = up->midx[r][k] - (r + 1);
        rc[(size_t)(w + r) * kUpSlots + k] = -up->mc[r][k];             // D+ right (mirror of D- left)
        ro[(size_t)(w + r) * kUpSlots + k] = (r + 1) - up->midx[r][k];
      }
    }
    rn[4 * w] = rn[4 * w + 1] = up->taps;
    for (int k = 0; k < up->taps; ++k) {
      rc[(size_t)(4 * w) * kUpSlots + k] = up->nbf[k];
      ro[(size_t)(4 * w) * kUpSlots + k] = up->of + k;
      rc[(size_t)(4 * w + 1) * kUpSlots + k] = up->nbb[k];
      ro[(size_t)(4 * w + 1) * kUpSlots + k] = up->ob + k;
    }
    double *drc;
    int *dro, *drn;
    CK(d->mem.get(&drc, rc.size()));
    CK(d->mem.get(&dro, ro.size()));
    CK(d->mem.get(&drn, rn.size()));
    CK(cudaMemcpyAsync(drc, rc.data(), sizeof(double) * rc.size(), cudaMemcpyHostToDevice, d->stream));
    CK(cudaMemcpyAsync(dro, ro.data(), sizeof(int) * ro.size(), cudaMemcpyHostToDevice, d->stream));
    CK(cudaMemcpyAsync(drn, rn.data(), sizeof(int) * rn.size(), cudaMemcpyHostToDevice, d->stream));
    CK(cudaStreamSynchronize(d->stream));
    b.urowc = drc;
    b.urowo = dro;
    b.urown = drn;
    b.uw = w;
    b.utaps = up->taps;
    b.uof = up->of;
    b.uob = up->ob;
    // strict-interior coefficients over h
    const double hh[3] = {1.0 / (double)(h.nq - 1), 1.0 / (double)(h.nr - 1), 1.0 / (double)(nsg - 1)};
    for (int a = 0; a < 3; ++a)
      for (int k = 0; k < up->taps; ++k) {
        b.ufw[a][k] = (T)(up->inf[k] / hh[a]);
        b.ubw[a][k] = (T)(up->inb[k] / hh[a]);
      }
  }
  // strict interior bounds, src/JU_xJU_yJU_z6.f90:16158-16173 (traditional-6,
  // width 6), :17915-17931 (upwind-4, width 4), src/RHS_Interior.f90:614-630
  // (upwind-6, 6) and :1218-1234 (upwind-DRP-6, 8)
  int np = bd.npml;
  const int w = upwind_table(b.fd) ? upwind_table(b.fd)->width : 6;
  int ix = bd.pml[0] ? std::max(np, w) : w, fx = bd.pml[1] ? std::max(np, w) : w;
  int iy = bd.pml[2] ? std::max(np, w) : w, fy = bd.pml[3] ? std::max(np, w) : w;
  int iz = bd.pml[4] ? std::max(np, w) : w, fz = bd.pml[5] ? std::max(np, w) : w;
  if (b.open_lo[2]) iz = 0;   // open faces: the central row reaches the face
  if (b.open_hi[2]) fz = 0;
  b.lo[0] = ix + 1; b.hi[0] = h.nq - fx;
  b.lo[1] = iy + 1; b.hi[1] = h.nr - fy;
  b.lo[2] = iz + 1; b.hi[2] = h.ns - fz;

  Alloc &M = d->mem;
  CK(M.get(&b.F0, 9 * vol));
  CK(M.get(&b.F1, 9 * vol));
  CK(M.get(&b.DF, 9 * vol));
  CK(M.get(&b.M, 3 * vol));
  if (d->fp32) CK(M.get(&b.FC, 9 * vol));
  if (bd.mesh == WQL3D_MESH_CURVILINEAR) CK(M.get(&b.G, 18 * vol, false));
  if (bd.mesh == WQL3D_MESH_CURVILINEAR && d->response != 0) CK(M.get(&b.S6, 6 * vol, false));
  if (bd.mesh == WQL3D_MESH_CURVILINEAR) {
    // face-SAT buffers of the lean path: faces with a physical boundary condition
    int off = 0;
    for (int f = 0; f < 6; ++f) {
      const int axis = f / 2;
      const int fn = axis == 0 ? h.nr * h.ns : axis == 1 ? h.nq * h.ns : h.nq * h.nr;
      b.foff[f] = off;
      b.fsat[f] = nullptr;
      b.fdq[f] = nullptr;
      if (bd.bc[f] > 0) {
        CK(M.get(&b.fsat[f], (size_t)9 * fn, false));
        if (bd.pml[f] && bd.npml > 0) CK(M.get(&b.fdq[f], (size_t)9 * fn, false));
        off += fn;
      }
    }
    b.foff[6] = off;
  }
  {
    // rates start at the reference's 1e40 sentinel (src/fields.f90:39) in FP64;
    // the first stage scales them by A(1) = 0.  FP32 cannot hold 1e40: zero.
    std::vector<T> init((size_t)9 * vol, (T)0);
    if (!d->fp32) {
      for (int c = 0; c < 9; ++c)
        for (int z = 1; z <= h.ns; ++z)
          for (int y = 1; y <= h.nr; ++y)
            for (int x = 1; x <= h.nq; ++x)
              init[(size_t)(c * vol + b.o1 + (x - 1) + b.sy * (y - 1) + b.sz * (z - 1))] = (T)1.0e40;
    }
    CK(cudaMemcpyAsync(b.DF, init.data(), sizeof(T) * 9 * vol, cudaMemcpyHostToDevice, d->stream));
    CK(cudaStreamSynchronize(d->stream));
  }
  int rc = put_array<T>(d, h, b.M, 3, bd.material, bd.host_nb);
  if (rc) return rc;

  // coordinates (host copy for lookups)
  std::vector<double> ghost;   // s-slab: coordinates of the 3 planes beyond each side, (3, 6, nr, nq)
  long long n1 = (long long)h.nq * h.nr * h.ns;
  h.coords.assign((size_t)(3 * n1), 0.0);
  if (bd.mesh == WQL3D_MESH_CARTESIAN) {
    double bh[3];
    int nn[3] = {h.nq, h.nr, nsg};
    for (int c = 0; c < 3; ++c) bh[c] = (bd.bqrs[c] - bd.aqrs[c]) / (double)(nn[c] - 1);
    for (int z = 1; z <= h.ns; ++z)
      for (int y = 1; y <= h.nr; ++y)
        for (int x = 1; x <= h.nq; ++x) {
          long long i = (x - 1) + (long long)h.nq * ((y - 1) + (long long)h.nr * (z - 1));
          h.coords[i] = bd.aqrs[0] + (double)(x - 1) * bh[0];
          h.coords[n1 + i] = bd.aqrs[1] + (double)(y - 1) * bh[1];
          h.coords[2 * n1 + i] = bd.aqrs[2] + (double)(z0 + z - 1) * bh[2];
        }
    if (slab) {
      // the 3 planes below and above the slab, for the metric's central rows
      const long long pl = (long long)h.nq * h.nr;
      ghost.assign((size_t)(3 * 6 * pl), 0.0);
      for (int k = 0; k < 6; ++k) {
        const int zg = k < 3 ? z0 - 2 + k : z0 + h.ns + 1 + (k - 3);
        for (int y = 1; y <= h.nr; ++y)
          for (int x = 1; x <= h.nq; ++x) {
            long long i = (x - 1) + (long long)h.nq * (y - 1) + pl * k;
            ghost[i] = bd.aqrs[0] + (double)(x - 1) * bh[0];
            ghost[6 * pl + i] = bd.aqrs[1] + (double)(y - 1) * bh[1];
            ghost[12 * pl + i] = bd.aqrs[2] + (double)(zg - 1) * bh[2];
          }
      }
    }
    // per-axis metric of the separable Cartesian mesh: 1 / (D6 x)(i), with
    // the SBP operator applied to the coordinate line exactly as
    // src/grid.f90:398-471 does (row-4 literal included)
    for (int a = 0; a < 3; ++a) {
      const int off = a == 2 ? z0 : 0;   // global index of the slab's planes
      const int nl = a == 0 ? h.nq : a == 1 ? h.nr : h.ns;
      std::vector<T> m((size_t)nl + 1, (T)0);
      double hh = 1.0 / (double)(nn[a] - 1);
      for (int i = 1; i <= nl; ++i) {
        int cnt, idx[8];
        double c[8];
        host_row(i + off, nn[a], b.lit, cnt, idx, c);
        double s = 0.0;
        for (int k = 0; k < cnt; ++k) s = s + c[k] * (bd.aqrs[a] + (double)(idx[k] - 1) * bh[a]);
        double Xa = (1.0 / hh) * s;
        m[(size_t)i] = (T)(1.0 / Xa);
      }
      T *dm;
      CK(M.get(&dm, m.size()));
      CK(cudaMemcpyAsync(dm, m.data(), sizeof(T) * m.size(), cudaMemcpyHostToDevice, d->stream));
      if (a == 0) b.mq = dm; else if (a == 1) b.mr = dm; else b.ms = dm;
    }
  } else {
    long long hn = (long long)(h.nq + 2 * bd.host_nb) * (h.nr + 2 * bd.host_nb) * (h.ns + 2 * bd.host_nb);
    for (int c = 0; c < 3; ++c)
      for (int z = 1; z <= h.ns; ++z)
        for (int y = 1; y <= h.nr; ++y)
          for (int x = 1; x <= h.nq; ++x) {
            int H = bd.host_nb;
            long long hi = (x - 1 + H) + (long long)(h.nq + 2 * H) * ((y - 1 + H) + (long long)(h.nr + 2 * H) * (z - 1 + H));
            h.coords[c * n1 + (x - 1) + (long long)h.nq * ((y - 1) + (long long)h.nr * (z - 1))] = bd.coords[c * hn + hi];
          }
    if (slab && (b.open_lo[2] || b.open_hi[2])) {
      if (!d->desc.slab_ghost_coords) return fail(WQL3D_EINVAL, "curvilinear slab needs slab_ghost_coords");
      ghost.assign(d->desc.slab_ghost_coords, d->desc.slab_ghost_coords + (size_t)3 * 6 * h.nq * h.nr);
    }
  }
  {
    // full metric and Jacobian of both mesh kinds from the coordinates
    // (the near-boundary operator and the face SATs use all nine entries)
    double *Xd, *metd, *Jd;
    CK(M.get(&Xd, 3 * vol));
    CK(M.get(&metd, 9 * vol));
    CK(M.get(&Jd, vol));
    rc = put_array<double>(d, h, Xd, 3, h.coords.data(), 0);
    if (rc) return rc;
    if (!ghost.empty()) {
      // ghost planes of the open sides (device planes -2..0 and ns+1..ns+3)
      for (int side = 0; side < 2; ++side) {
        if (!(side ? b.open_hi[2] : b.open_lo[2])) continue;
        for (int c = 0; c < 3; ++c) {
          cudaMemcpy3DParms q;
          memset(&q, 0, sizeof(q));
          q.srcPtr = make_cudaPitchedPtr((void *)(ghost.data() + (size_t)c * 6 * h.nq * h.nr), (size_t)h.nq * sizeof(double),
                                         h.nq, h.nr);
          q.srcPos = make_cudaPos(0, 0, side ? 3 : 0);
          q.dstPtr = make_cudaPitchedPtr((void *)(Xd + (long long)c * vol), (size_t)h.PX * sizeof(double), h.PX, h.PY);
          q.dstPos = make_cudaPos((size_t)h.XOFF * sizeof(double), NB, side ? NB + h.ns : 0);
          q.extent = make_cudaExtent((size_t)h.nq * sizeof(double), h.nr, 3);
          q.kind = cudaMemcpyHostToDevice;
          CK(cudaMemcpy3DAsync(&q, d->stream));
        }
      }
      CK(cudaStreamSynchronize(d->stream));
    }
    b.X = Xd;
    b.mms = d->desc.mms ? 1 : 0;
    if (b.mms) {
      const double pi = 3.141592653589793;
      b.mms_k[0] = d->desc.mms_nt * pi;
      b.mms_k[1] = d->desc.mms_nx * pi;
      b.mms_k[2] = d->desc.mms_ny * pi;
      b.mms_k[3] = d->desc.mms_nz * pi;
    }
    dim3 th(32, 4, 2), gr((h.nq + 31) / 32, (h.nr + 3) / 4, (h.ns + 1) / 2);
    k_metrics<T><<<gr, th, 0, d->stream>>>(b, Xd, metd, Jd);
    CK(cudaGetLastError());
    if (sizeof(T) == sizeof(double)) {
      b.met = (const T *)metd;
      b.J = (const T *)Jd;
    } else {
      T *mt, *jt;
      CK(M.get(&mt, 9 * vol));
      CK(M.get(&jt, vol));
      k_convert<T><<<1024, 256, 0, d->stream>>>(metd, mt, 9 * vol);
      k_convert<T><<<1024, 256, 0, d->stream>>>(Jd, jt, vol);
      b.met = mt;
      b.J = jt;
    }
    // face bases from the device metrics (src/unit_normals.f90:8-160)
    std::vector<double> met9((size_t)9 * vol);
    CK(cudaMemcpyAsync(met9.data(), metd, sizeof(double) * 9 * vol, cudaMemcpyDeviceToHost, d->stream));
    CK(cudaStreamSynchronize(d->stream));
    for (int f = 0; f < 6; ++f) {
      int axis = f / 2;
      int d0 = axis == 0 ? h.nr : h.nq, d1 = axis == 2 ? h.nr : h.ns;
      long long fn = (long long)d0 * d1;
      std::vector<T> basis((size_t)(9 * fn));
      int fixed = (f % 2 == 0) ? 1 : (axis == 0 ? h.nq : axis == 1 ? h.nr : h.ns);
      for (int c2 = 1; c2 <= d1; ++c2)
        for (int c1 = 1; c1 <= d0; ++c1) {
          int x, y, z;
          if (axis == 0) { x = fixed; y = c1; z = c2; }
          else if (axis == 1) { x = c1; y = fixed; z = c2; }
          else { x = c1; y = c2; z = fixed; }
          long long p = b.o1 + (x - 1) + b.sy * (y - 1) + b.sz * (z - 1);
          double qx = met9[(size_t)((0 + axis) * vol + p)], qy = met9[(size_t)((3 + axis) * vol + p)],
                 qz = met9[(size_t)((6 + axis) * vol + p)];
          double norm = sqrt(qx * qx + qy * qy + qz * qz);
          double n3[3] = {qx / norm, qy / norm, qz / norm}, l3[3], m3[3];
          gen_orth(l3, m3, n3);
          long long fp = (c1 - 1) + (long long)d0 * (c2 - 1);
          for (int c = 0; c < 3; ++c) {
            basis[(size_t)((0 + c) * fn + fp)] = (T)l3[c];
            basis[(size_t)((3 + c) * fn + fp)] = (T)m3[c];
            basis[(size_t)((6 + c) * fn + fp)] = (T)n3[c];
          }
        }
      T *dbase;
      CK(M.get(&dbase, basis.size()));
      CK(cudaMemcpyAsync(dbase, basis.data(), sizeof(T) * basis.size(), cudaMemcpyHostToDevice, d->stream));
      CK(cudaStreamSynchronize(d->stream));
      b.nrm[f] = dbase;
    }
    // a Cartesian block whose off-diagonal metric entries are roundoff
    // (|off| <= 1e-12 |diag|; a single-precision row-4 literal gives ~1e-9) takes the separable near-boundary path
    if (bd.mesh == WQL3D_MESH_CARTESIAN) {
      double dmin = 1e300, omax = 0.0;
      for (int z = 1; z <= h.ns; ++z)
        for (int y = 1; y <= h.nr; ++y)
          for (int x = 1; x <= h.nq; ++x) {
            long long p = b.o1 + (x - 1) + b.sy * (y - 1) + b.sz * (z - 1);
            for (int r = 0; r < 3; ++r)
              for (int c = 0; c < 3; ++c) {
                double v = fabs(met9[(size_t)((r * 3 + c) * vol + p)]);
                if (r == c) dmin = std::min(dmin, v);
                else omax = std::max(omax, v);
              }
          }
      b.sep = (omax <= 1e-12 * dmin && b.fd == WQL3D_FD_TRADITIONAL6) ? 1 : 0;
    }
  }

  // PML slabs, src/pml.f90:11-168
  b.npml = np;
  b.d0 = (T)(6.0 / (2.0 * 1.0) * log(1.0 / 1.0e-3));
  for (int f = 0; f < 6; ++f) {
    b.pml_on[f] = (bd.pml[f] && np > 0) ? 1 : 0;
    int *B = b.pb[f];
    B[0] = 1; B[1] = h.nq; B[2] = 1; B[3] = h.nr; B[4] = 1; B[5] = h.ns;
    if (!b.pml_on[f]) continue;
    switch (f) {
      case 0: B[1] = np; break;
      case 1: B[0] = h.nq - np + 1; break;
      case 2: B[3] = np; break;
      case 3: B[2] = h.nr - np + 1; break;
      case 4: B[5] = np; break;
      default: B[4] = h.ns - np + 1; break;
    }
    long long pv = (long long)(B[1] - B[0] + 1) * (B[3] - B[2] + 1) * (B[5] - B[4] + 1);
    b.pvol[f] = pv;
    CK(M.get(&b.Q[f], 9 * pv));
    CK(M.get(&b.DQ[f], 9 * pv));
    std::vector<T> init((size_t)(9 * pv), d->fp32 ? (T)0 : (T)1.0e40);  // DQ = 1e40, src/pml.f90
    CK(cudaMemcpyAsync(b.DQ[f], init.data(), sizeof(T) * init.size(), cudaMemcpyHostToDevice, d->stream));
    CK(cudaStreamSynchronize(d->stream));
  }

  // anelastic memory variables
  b.nmech = d->nmech;
  if (d->nmech) {
    CK(M.get(&b.eta, (size_t)6 * d->nmech * vol));
    CK(M.get(&b.deta, (size_t)6 * d->nmech * vol));
    for (int i = 0; i < 8; ++i) {
      b.tau[i] = (T)d->desc.tau[i];
      b.itau[i] = (T)(1.0 / d->desc.tau[i]);
      b.w[i] = (T)d->desc.weight[i];
      b.ss[i] = (T)d->desc.strength_s[i];
      b.ps[i] = (T)d->desc.strength_p[i];
    }
    b.coarse = d->desc.coarse_grain;
    if (d->response != WQL3D_FQ8) {
      T *qs, *qp;
      CK(M.get(&qs, vol));
      CK(M.get(&qp, vol));
      std::vector<double> tmp;
      const double *qsh = bd.qs_inv, *qph = bd.qp_inv;
      int hnb = bd.host_nb;
      long long hn = (long long)(h.nq + 2 * hnb) * (h.nr + 2 * hnb) * (h.ns + 2 * hnb);
      std::vector<double> cs, cp;
      if (!qsh) { cs.assign((size_t)hn, 1.0 / d->desc.Qs0); qsh = cs.data(); }
      if (!qph) { cp.assign((size_t)hn, 1.0 / d->desc.Qp0); qph = cp.data(); }
      rc = put_array<T>(d, h, qs, 1, qsh, hnb);
      if (rc) return rc;
      rc = put_array<T>(d, h, qp, 1, qph, hnb);
      if (rc) return rc;
      CK(cudaStreamSynchronize(d->stream));
      b.qs = qs;
      b.qp = qp;
    }
  }

  // sources: nearest node (Find_Coordinates_moment) and support box
  h.nsrc = bd.nsrc;
  b.nsrc = bd.nsrc;
  b.src_order = bd.src_order;
  b.src_alpha = bd.src_alpha;
  b.src_half = bd.src_order == 4 ? 4 : 2;
  b.sbox[0] = b.sbox[2] = b.sbox[4] = 1 << 30;
  b.sbox[1] = b.sbox[3] = b.sbox[5] = -(1 << 30);
  if (bd.nsrc > 0) {
    if (!bd.src_type || !bd.src_par) return fail(WQL3D_EINVAL, "sources need src_type and src_par");
    std::vector<DevSource> ss((size_t)bd.nsrc);
    for (int i = 0; i < bd.nsrc; ++i) {
      DevSource &s = ss[(size_t)i];
      s.type = bd.src_type[i];
      for (int k = 0; k < 11; ++k) s.par[k] = bd.src_par[11 * i + k];
      nearest_moment(h, s.par[8], s.par[9], s.par[10], s.near);
      if (s.near[0] > 0) {
        long long ii = (s.near[0] - 1) + (long long)h.nq * ((s.near[1] - 1) + (long long)h.nr * (s.near[2] - 1));
        for (int c = 0; c < 3; ++c) s.phys[c] = h.coords[(size_t)(c * n1 + ii)];
        for (int c = 0; c < 3; ++c) {
          b.sbox[2 * c] = std::min(b.sbox[2 * c], s.near[c] - b.src_half);
          b.sbox[2 * c + 1] = std::max(b.sbox[2 * c + 1], s.near[c] + b.src_half);
        }
      } else {
        for (int c = 0; c < 3; ++c) s.phys[c] = -1.0;
      }
    }
    DevSource *ds;
    CK(M.get(&ds, ss.size()));
    CK(cudaMemcpyAsync(ds, ss.data(), sizeof(DevSource) * ss.size(), cudaMemcpyHostToDevice, d->stream));
    CK(cudaStreamSynchronize(d->stream));
    b.src = ds;
  }
  // receivers (Find_Coordinates)
  h.nrec = bd.nrec;
  b.nrec = bd.nrec;
  b.max_samples = d->desc.max_samples;
  if (bd.nrec > 0) {
    h.ridx.assign((size_t)3 * bd.nrec, -9999);
    for (int r = 0; r < bd.nrec; ++r)
      nearest_receiver(h, bd.rec_xyz[3 * r], bd.rec_xyz[3 * r + 1], bd.rec_xyz[3 * r + 2], &h.ridx[(size_t)3 * r]);
    int *ri;
    CK(M.get(&ri, h.ridx.size()));
    CK(cudaMemcpyAsync(ri, h.ridx.data(), sizeof(int) * h.ridx.size(), cudaMemcpyHostToDevice, d->stream));
    b.ridx = ri;
    CK(M.get(&b.seis, (size_t)std::max(1, b.max_samples) * bd.nrec * 4));
    CK(cudaStreamSynchronize(d->stream));
  }
  return WQL3D_OK;
}

template <typename T>
void launch_stage(wql3d_domain *d, int bi, const StageArgs &a, bool fused = false) {
  Blk<T> &b = blk<T>(d, bi);
  const int mesh = d->hb[bi].mesh;
  StageCtx c{d->stream, d->response, &d->launches, d->side, d->fork, d->join};
  const bool special = tuning().generic || b.mms || b.fd != WQL3D_FD_TRADITIONAL6;
  if (fused && mesh == WQL3D_MESH_CARTESIAN && a.flags == F_ALL && !special)
    launch_cart_stage<T>(b, c, a);
  else if (mesh == WQL3D_MESH_CURVILINEAR && b.G && !special)
    launch_curv_stage<T>(b, c, a);
  else
    launch_generic_stage<T>(b, mesh, c, a);
}

template <typename T>
int enqueue_stage(wql3d_domain *d, int stage, double dt, int flags, void *rec = nullptr) {
  StageArgs a;
  a.cur = d->cur;
  a.flags = flags;
  a.rec = rec;
  a.stage = stage;
  a.A = kRkA[stage - 1];
  a.Bdt = kRkB[stage - 1] * dt;
  a.dt = dt;
  a.time = d->time;
  if (d->has_iface && (flags & F_ISAT)) {
    // interface law, SAT vectors, DS = A DS + ... and S = S + B dt DS in one pass
    launch_iface<T>(d->iface, blk<T>(d, 0), blk<T>(d, 1), a, d->stream);
    d->launches++;
  }
  for (int i = 0; i < d->nblocks; ++i) launch_stage<T>(d, i, a, true);
  if (flags & F_UPDATE) d->cur ^= 1;
  return WQL3D_OK;
}

template <typename T>
int enqueue_sample(wql3d_domain *d, int w_stride) {
  int last = -1;
  for (int i = 0; i < d->nblocks; ++i)
    if (d->hb[i].nrec > 0) last = i;
  for (int i = 0; i < d->nblocks; ++i) {
    if (d->hb[i].nrec <= 0) continue;
    k_sample<T><<<1, 256, 0, d->stream>>>(blk<T>(d, i), d->cur, d->time, w_stride, i == last ? 1 : 0);
    d->launches++;
  }
  return WQL3D_OK;
}

template <typename T>
int enqueue_step(wql3d_domain *d, double dt, int w_stride) {
  enqueue_sample<T>(d, w_stride);
  for (int s = 1; s <= 5; ++s) {
    int rc = enqueue_stage<T>(d, s, dt, F_ALL);
    if (rc) return rc;
  }
  k_advance<<<1, 32, 0, d->stream>>>(d->time, dt);
  d->launches++;
  return WQL3D_OK;
}

template <typename T>
int run_steps(wql3d_domain *d, double dt, int nsteps, int w_stride) {
  // CUDA graph of two steps (five stages each, so the field-buffer parity
  // returns to its start) replayed nsteps/2 times
  int pairs = nsteps / 2;
  if (pairs > 0) {
    if (!d->graph || d->g_dt != dt || d->g_w != w_stride || d->g_cur != d->cur) {
      if (d->graph) { cudaGraphExecDestroy(d->graph); d->graph = nullptr; }
      int cur0 = d->cur;
      int64_t l0 = d->launches;
      cudaGraph_t g;
      CK(cudaStreamBeginCapture(d->stream, cudaStreamCaptureModeThreadLocal));
      enqueue_step<T>(d, dt, w_stride);
      enqueue_step<T>(d, dt, w_stride);
      CK(cudaStreamEndCapture(d->stream, &g));
      CK(cudaGraphInstantiate(&d->graph, g, 0));
      cudaGraphDestroy(g);
      d->cur = cur0;
      d->g_dt = dt;
      d->g_w = w_stride;
      d->g_cur = cur0;
      d->g_launches = d->launches - l0;
      d->launches = l0;
    }
    const int64_t per_pair = d->g_launches;
    for (int k = 0; k < pairs; ++k) {
      CK(cudaGraphLaunch(d->graph, d->stream));
      d->launches += per_pair;
    }
  }
  if (nsteps % 2) {
    int rc = enqueue_step<T>(d, dt, w_stride);
    if (rc) return rc;
  }
  CK(cudaGetLastError());
  return WQL3D_OK;
}

template <typename T>
int final_state(wql3d_domain *d, double *maxF, double *maxEta, double *bmax) {
  double mf = 0.0, me = 0.0;
  int nonfinite = 0;
  for (int i = 0; i < d->nblocks; ++i) {
    Blk<T> &b = blk<T>(d, i);
    const T *F = d->cur ? b.F1 : b.F0;
    CK(cudaMemsetAsync(d->flag, 0, sizeof(int), d->stream));
    k_maxabs<T><<<592, 256, 0, d->stream>>>(F, 9 * b.vol, d->red, d->flag);
    d->launches++;
    std::vector<double> part(592);
    int fl = 0;
    CK(cudaMemcpyAsync(part.data(), d->red, sizeof(double) * 592, cudaMemcpyDeviceToHost, d->stream));
    CK(cudaMemcpyAsync(&fl, d->flag, sizeof(int), cudaMemcpyDeviceToHost, d->stream));
    CK(cudaStreamSynchronize(d->stream));
    double m = 0.0;
    for (double v : part) m = std::max(m, v);
    nonfinite |= fl;
    if (bmax) bmax[i] = m;
    mf = std::max(mf, m);
    if (b.nmech) {
      CK(cudaMemsetAsync(d->flag, 0, sizeof(int), d->stream));
      k_maxabs<T><<<592, 256, 0, d->stream>>>(b.eta, (long long)6 * b.nmech * b.vol, d->red, d->flag);
      d->launches++;
      CK(cudaMemcpyAsync(part.data(), d->red, sizeof(double) * 592, cudaMemcpyDeviceToHost, d->stream));
      CK(cudaMemcpyAsync(&fl, d->flag, sizeof(int), cudaMemcpyDeviceToHost, d->stream));
      CK(cudaStreamSynchronize(d->stream));
      for (double v : part) me = std::max(me, v);
      nonfinite |= fl;
    }
  }
  if (maxF) *maxF = mf;
  if (maxEta) *maxEta = me;
  if (nonfinite) return fail(WQL3D_ENONFINITE, "non-finite field or memory state (RUN-ELASTIC-001 / RUN-Q*-001)");
  return WQL3D_OK;
}

wql3d_domain *checked(wql3d_domain *d) { return d; }

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
// v_z of block bi set to v everywhere (the current field buffer)
void init_velocity(wql3d_domain *d, int bi, double v) {
  const long long np = (long long)d->hb[bi].nq * d->hb[bi].nr * d->hb[bi].ns;
  const unsigned gr = (unsigned)((np + 255) / 256);
  if (d->fp32) k_fill_component<float><<<gr, 256, 0, d->stream>>>(d->bf[bi], d->cur ? d->bf[bi].F1 : d->bf[bi].F0, 2, (float)v);
  else k_fill_component<double><<<gr, 256, 0, d->stream>>>(d->bd[bi], d->cur ? d->bd[bi].F1 : d->bd[bi].F0, 2, v);
}

// ghost-plane pack / unpack of an s-slab domain on its stream
template <typename T>
int halo_launch(wql3d_domain *d, Blk<T> &b, int kind, int unpack) {
  T *buf = (T *)(unpack ? d->halo_recv : d->halo_send);
  const int ncomp = kind == WQL3D_HALO_FIELDS ? 9 : 10;
  T *a0 = kind == WQL3D_HALO_FIELDS ? (d->cur ? b.F1 : b.F0) : const_cast<T *>(b.met);
  T *a1 = kind == WQL3D_HALO_FIELDS ? a0 : const_cast<T *>(b.J);
  const int n0 = 9;
  const long long n = (long long)2 * ncomp * 3 * b.nx * b.ny;
  k_halo<T><<<(unsigned)((n + 255) / 256), 256, 0, d->stream>>>(b, buf, a0, n0, a1, ncomp, unpack);
  d->launches++;
  CK(cudaGetLastError());
  return WQL3D_OK;
}

extern "C" {

const char *wql3d_last_error(void) { return g_err.c_str(); }

int wql3d_domain_create(const wql3d_domain_desc *desc, wql3d_domain **out) {
  if (!desc || !out) return fail(WQL3D_EINVAL, "null argument");
  *out = nullptr;
  if (desc->abi_version != WQL3D_ABI_VERSION) return fail(WQL3D_EINVAL, "ABI version mismatch");
  if (desc->nblocks < 1 || desc->nblocks > 2) return fail(WQL3D_EINVAL, "nblocks must be 1 or 2");
  if (desc->precision != WQL3D_FP64 && desc->precision != WQL3D_FP32_COMPENSATED) return fail(WQL3D_EINVAL, "precision");
  if (desc->response < 0 || desc->response > 3) return fail(WQL3D_EINVAL, "response");
  int dev_count = 0;
  if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) return fail(WQL3D_ECUDA, "no CUDA device");
  int rc = upload_constants();
  if (rc) return rc;
  wql3d_domain *d = new wql3d_domain();
  d->desc = *desc;
  d->nblocks = desc->nblocks;
  d->fp32 = desc->precision == WQL3D_FP32_COMPENSATED;
  d->response = desc->response;
  d->nmech = desc->response == WQL3D_ELASTIC ? 0 : desc->response == WQL3D_Q4 ? 4 : 8;
  if (cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete d;
    return fail(WQL3D_ECUDA, "stream creation failed");
  }
  d->mem.stream = d->stream;
  auto cleanup = [&](int code) {
    cudaStreamSynchronize(d->stream);
    d->mem.release();
    if (d->side) cudaStreamDestroy(d->side);
    if (d->fork) cudaEventDestroy(d->fork);
    if (d->join) cudaEventDestroy(d->join);
    cudaStreamDestroy(d->stream);
    delete d;
    return code;
  };
  if (cudaStreamCreateWithFlags(&d->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&d->fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&d->join, cudaEventDisableTiming) != cudaSuccess)
    return cleanup(fail(WQL3D_ECUDA, "side stream creation failed"));
  if (d->mem.get(&d->time, 1) != cudaSuccess) return cleanup(fail(WQL3D_ENOMEM, "time"));
  DevTime t0 = {0.0, 1, 0, 0, 0};
  if (cudaMemcpyAsync(d->time, &t0, sizeof(t0), cudaMemcpyHostToDevice, d->stream) != cudaSuccess ||
      cudaStreamSynchronize(d->stream) != cudaSuccess)
    return cleanup(fail(WQL3D_ECUDA, "time init"));
  if (d->mem.get(&d->red, 592) != cudaSuccess || d->mem.get(&d->flag, 1) != cudaSuccess)
    return cleanup(fail(WQL3D_ENOMEM, "reduction scratch"));
  for (int i = 0; i < desc->nblocks; ++i) {
    const long long nq = desc->block[i].nq, nr = desc->block[i].nr, ns = desc->block[i].ns;
    d->plane_cap = std::max(d->plane_cap, 9 * std::max(nq * nr, std::max(nq * ns, nr * ns)));
  }
  if (d->mem.get(&d->plane, (size_t)d->plane_cap, false) != cudaSuccess)
    return cleanup(fail(WQL3D_ENOMEM, "plane buffer"));
  for (int i = 0; i < desc->nblocks; ++i) {
    const long long nq = desc->block[i].nq + 6, nr = desc->block[i].nr + 6, ns = desc->block[i].ns + 6;
    d->xfer_cap = std::max(d->xfer_cap, 9 * nq * nr * ns);
  }
  if (d->mem.get(&d->xfer, (size_t)d->xfer_cap, false) != cudaSuccess)
    return cleanup(fail(WQL3D_ENOMEM, "transfer staging buffer"));
  for (int i = 0; i < desc->nblocks; ++i) {
    const int fd = desc->block[i].fd_operator;
    if (fd < WQL3D_FD_TRADITIONAL6 || fd > WQL3D_FD_UPWIND_DRP6)
      return cleanup(fail(WQL3D_EINVAL, "unknown fd_operator"));
    if (fd != WQL3D_FD_TRADITIONAL6 && desc->slab_ns_global > 0)
      return cleanup(fail(WQL3D_EINVAL, "upwind blocks are not split into s-slabs"));
  }
  if (desc->slab_ns_global > 0) {
    // one s-slab of a larger block: open faces carry no boundary condition or PML
    const wql3d_block_desc &b0 = desc->block[0];
    if (desc->nblocks != 1 || desc->remote_side != 0 || desc->mms)
      return cleanup(fail(WQL3D_EINVAL, "an s-slab domain holds one block without interface or MMS"));
    if (desc->slab_z0 < 0 || desc->slab_z0 + b0.ns > desc->slab_ns_global)
      return cleanup(fail(WQL3D_EINVAL, "slab planes outside the block"));
    d->slab = true;
    if (desc->slab_z0 > 0) { d->desc.block[0].bc[4] = 0; d->desc.block[0].pml[4] = 0; }
    if (desc->slab_z0 + b0.ns < desc->slab_ns_global) { d->desc.block[0].bc[5] = 0; d->desc.block[0].pml[5] = 0; }
    for (int f = 4; f < 6; ++f)
      if (d->desc.block[0].pml[f] && b0.npml > b0.ns)
        return cleanup(fail(WQL3D_EINVAL, "an s-face PML slab must lie inside one slab"));
    const size_t hn = (size_t)2 * 10 * 3 * b0.nq * b0.nr;
    const size_t eb = d->fp32 ? sizeof(float) : sizeof(double);
    if (d->mem.get((char **)&d->halo_send, hn * eb) != cudaSuccess ||
        d->mem.get((char **)&d->halo_recv, hn * eb) != cudaSuccess)
      return cleanup(fail(WQL3D_ENOMEM, "halo buffers"));
  }
  for (int i = 0; i < d->nblocks; ++i) {
    rc = d->fp32 ? setup_block<float>(d, i) : setup_block<double>(d, i);
    if (rc) return cleanup(rc);
  }
  if (d->nblocks == 1 && d->desc.remote_side != 0) {
    const int side = d->desc.remote_side;
    rc = d->fp32 ? setup_iface_remote<float>(d->iface, d->desc, d->bf[0], d->hb[0].coords, side, d->mem, d->stream)
                 : setup_iface_remote<double>(d->iface, d->desc, d->bd[0], d->hb[0].coords, side, d->mem, d->stream);
    if (rc) return cleanup(fail(rc, "remote interface setup failed"));
    d->has_iface = true;
    if (d->fp32) d->bf[0].isat[side == 1 ? 1 : 0] = (float *)(side == 1 ? d->iface.sat_m : d->iface.sat_p);
    else d->bd[0].isat[side == 1 ? 1 : 0] = (double *)(side == 1 ? d->iface.sat_m : d->iface.sat_p);
    // init_vel_state: v_z = -Vin/2 on block 1's rank, +Vin/2 on block 2's (src/domain.f90:273-274)
    if (rs_problem(d->desc.fault_problem)) init_velocity(d, 0, side == 1 ? -0.5e-12 : 0.5e-12);
  } else if (d->desc.remote_side != 0) {
    return cleanup(fail(WQL3D_EINVAL, "remote_side needs nblocks = 1"));
  }
  if (d->nblocks == 2) {
    rc = d->fp32 ? setup_iface<float>(d->iface, d->desc, d->bf[0], d->bf[1], d->hb[0].coords, d->hb[1].coords,
                                      d->mem, d->stream)
                 : setup_iface<double>(d->iface, d->desc, d->bd[0], d->bd[1], d->hb[0].coords, d->hb[1].coords,
                                       d->mem, d->stream);
    if (rc) return cleanup(fail(rc, "interface setup failed"));
    d->has_iface = true;
    if (d->fp32) { d->bf[0].isat[1] = (float *)d->iface.sat_m; d->bf[1].isat[0] = (float *)d->iface.sat_p; }
    else { d->bd[0].isat[1] = (double *)d->iface.sat_m; d->bd[1].isat[0] = (double *)d->iface.sat_p; }
    // init_vel_state of the one-process run: block 1's v_z = -Vin/2 (src/domain.f90:273)
    if (rs_problem(d->desc.fault_problem)) init_velocity(d, 0, -0.5e-12);
  }
  if (cudaStreamSynchronize(d->stream) != cudaSuccess || cudaGetLastError() != cudaSuccess)
    return cleanup(fail(WQL3D_ECUDA, "setup kernels failed"));
  *out = d;
  return WQL3D_OK;
}

int wql3d_domain_destroy(wql3d_domain *d) {
  if (!d) return WQL3D_OK;
  cudaStreamSynchronize(d->stream);
  if (d->side) cudaStreamSynchronize(d->side);
  if (d->graph) cudaGraphExecDestroy(d->graph);
  d->mem.release();
  if (d->side) cudaStreamDestroy(d->side);
  if (d->fork) cudaEventDestroy(d->fork);
  if (d->join) cudaEventDestroy(d->join);
  cudaStreamDestroy(d->stream);
  delete d;
  return WQL3D_OK;
}

#define DOM_CHECK(d, bi)                                                         \
  if (!(d)) return fail(WQL3D_EINVAL, "null domain");                            \
  if ((bi) < 0 || (bi) >= (d)->nblocks) return fail(WQL3D_EINVAL, "block index");

int wql3d_set_fields(wql3d_domain *d, int bi, const double *F, int32_t host_nb) {
  DOM_CHECK(d, bi);
  if (!F || host_nb < 0) return fail(WQL3D_EINVAL, "fields");
  int rc = d->fp32 ? put_array<float>(d, d->hb[bi], d->cur ? d->bf[bi].F1 : d->bf[bi].F0, 9, F, host_nb)
                   : put_array<double>(d, d->hb[bi], d->cur ? d->bd[bi].F1 : d->bd[bi].F0, 9, F, host_nb);
  if (rc) return rc;
  if (d->fp32) CK(cudaMemsetAsync(d->bf[bi].FC, 0, sizeof(float) * 9 * d->bf[bi].vol, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  return WQL3D_OK;
}

int wql3d_get_fields(wql3d_domain *d, int bi, double *F, int32_t host_nb) {
  DOM_CHECK(d, bi);
  if (!F || host_nb < 0) return fail(WQL3D_EINVAL, "fields");
  if (host_nb > 0) {
    long long hn = (long long)(d->hb[bi].nq + 2 * host_nb) * (d->hb[bi].nr + 2 * host_nb) * (d->hb[bi].ns + 2 * host_nb);
    memset(F, 0, sizeof(double) * 9 * hn);
  }
  return d->fp32 ? get_array<float>(d, d->hb[bi], d->cur ? d->bf[bi].F1 : d->bf[bi].F0, 9, F, host_nb)
                 : get_array<double>(d, d->hb[bi], d->cur ? d->bd[bi].F1 : d->bd[bi].F0, 9, F, host_nb);
}

int wql3d_set_rates(wql3d_domain *d, int bi, const double *DF, int32_t host_nb) {
  DOM_CHECK(d, bi);
  if (!DF || host_nb < 0) return fail(WQL3D_EINVAL, "rates");
  int rc = d->fp32 ? put_array<float>(d, d->hb[bi], d->bf[bi].DF, 9, DF, host_nb)
                   : put_array<double>(d, d->hb[bi], d->bd[bi].DF, 9, DF, host_nb);
  if (rc) return rc;
  CK(cudaStreamSynchronize(d->stream));
  return WQL3D_OK;
}

int wql3d_get_rates(wql3d_domain *d, int bi, double *DF, int32_t host_nb) {
  DOM_CHECK(d, bi);
  if (!DF || host_nb < 0) return fail(WQL3D_EINVAL, "rates");
  if (host_nb > 0) {
    long long hn = (long long)(d->hb[bi].nq + 2 * host_nb) * (d->hb[bi].nr + 2 * host_nb) * (d->hb[bi].ns + 2 * host_nb);
    memset(DF, 0, sizeof(double) * 9 * hn);
  }
  return d->fp32 ? get_array<float>(d, d->hb[bi], d->bf[bi].DF, 9, DF, 0 + host_nb)
                 : get_array<double>(d, d->hb[bi], d->bd[bi].DF, 9, DF, host_nb);
}

int wql3d_get_memory_variables(wql3d_domain *d, int bi, double *eta) {
  DOM_CHECK(d, bi);
  if (!d->nmech) return fail(WQL3D_EINVAL, "elastic domain has no memory variables");
  return d->fp32 ? get_array<float>(d, d->hb[bi], d->bf[bi].eta, 6 * d->nmech, eta, 0)
                 : get_array<double>(d, d->hb[bi], d->bd[bi].eta, 6 * d->nmech, eta, 0);
}

int wql3d_get_metrics(wql3d_domain *d, int bi, double *out) {
  DOM_CHECK(d, bi);
  const HostBlock &h = d->hb[bi];
  long long n1 = (long long)h.nq * h.nr * h.ns;
  if (h.mesh == WQL3D_MESH_CARTESIAN) {
    // diagonal metric and J of the separable mesh, off-diagonals zero
    int nn[3] = {h.nq, h.nr, h.ns};
    std::vector<double> m[3];
    for (int a = 0; a < 3; ++a) {
      m[a].resize((size_t)nn[a] + 1);
      const void *src = a == 0 ? (d->fp32 ? (const void *)d->bf[bi].mq : (const void *)d->bd[bi].mq)
                        : a == 1 ? (d->fp32 ? (const void *)d->bf[bi].mr : (const void *)d->bd[bi].mr)
                                 : (d->fp32 ? (const void *)d->bf[bi].ms : (const void *)d->bd[bi].ms);
      if (d->fp32) {
        std::vector<float> tmp((size_t)nn[a] + 1);
        CK(cudaMemcpyAsync(tmp.data(), src, sizeof(float) * tmp.size(), cudaMemcpyDeviceToHost, d->stream));
        CK(cudaStreamSynchronize(d->stream));
        for (size_t i = 0; i < tmp.size(); ++i) m[a][i] = tmp[i];
      } else {
        CK(cudaMemcpyAsync(m[a].data(), src, sizeof(double) * m[a].size(), cudaMemcpyDeviceToHost, d->stream));
        CK(cudaStreamSynchronize(d->stream));
      }
    }
    memset(out, 0, sizeof(double) * 10 * n1);
    for (int z = 1; z <= h.ns; ++z)
      for (int y = 1; y <= h.nr; ++y)
        for (int x = 1; x <= h.nq; ++x) {
          long long i = (x - 1) + (long long)h.nq * ((y - 1) + (long long)h.nr * (z - 1));
          out[0 * n1 + i] = m[0][x];
          out[4 * n1 + i] = m[1][y];
          out[8 * n1 + i] = m[2][z];
          out[9 * n1 + i] = 1.0 / (m[0][x] * m[1][y] * m[2][z]);
        }
    return WQL3D_OK;
  }
  int rc = d->fp32 ? get_array<float>(d, h, d->bf[bi].met, 9, out, 0) : get_array<double>(d, h, d->bd[bi].met, 9, out, 0);
  if (rc) return rc;
  return d->fp32 ? get_array<float>(d, h, d->bf[bi].J, 1, out + 9 * n1, 0) : get_array<double>(d, h, d->bd[bi].J, 1, out + 9 * n1, 0);
}

int wql3d_get_interface(wql3d_domain *d, double *out) {
  if (!d || !d->has_iface) return fail(WQL3D_EINVAL, "no interface");
  return iface_download(d->iface, out, d->stream);
}

int wql3d_get_fault_output(wql3d_domain *d, int kind, double *out) {
  if (!d || !d->has_iface) return fail(WQL3D_EINVAL, "no interface");
  if (!out) return fail(WQL3D_EINVAL, "null output");
  int rc = iface_fault_output(d->iface, kind, out, d->stream);
  if (rc) return fail(rc, "fault output kind " + std::to_string(kind));
  return WQL3D_OK;
}

int wql3d_set_time(wql3d_domain *d, double t) {
  if (!d) return fail(WQL3D_EINVAL, "null domain");
  DevTime h;
  CK(cudaMemcpyAsync(&h, d->time, sizeof(h), cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  h.t = t;
  CK(cudaMemcpyAsync(d->time, &h, sizeof(h), cudaMemcpyHostToDevice, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  return WQL3D_OK;
}

int wql3d_get_time(wql3d_domain *d, double *t) {
  if (!d || !t) return fail(WQL3D_EINVAL, "null argument");
  DevTime h;
  CK(cudaMemcpyAsync(&h, d->time, sizeof(h), cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  *t = h.t;
  return WQL3D_OK;
}

int wql3d_stage(wql3d_domain *d, int stage, double dt) {
  if (!d) return fail(WQL3D_EINVAL, "null domain");
  if (stage < 1 || stage > 5) return fail(WQL3D_EINVAL, "stage must be 1..5");
  int rc = d->fp32 ? enqueue_stage<float>(d, stage, dt, F_ALL) : enqueue_stage<double>(d, stage, dt, F_ALL);
  if (rc) return rc;
  if (stage == 5) {
    k_advance<<<1, 32, 0, d->stream>>>(d->time, dt);
    d->launches++;
  }
  CK(cudaGetLastError());
  return WQL3D_OK;
}

int wql3d_begin_step(wql3d_domain *d, int n, int w_stride) {
  if (!d) return fail(WQL3D_EINVAL, "null domain");
  DevTime h;
  CK(cudaMemcpyAsync(&h, d->time, sizeof(h), cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  h.n = n;
  CK(cudaMemcpyAsync(d->time, &h, sizeof(h), cudaMemcpyHostToDevice, d->stream));
  int rc = d->fp32 ? enqueue_sample<float>(d, w_stride) : enqueue_sample<double>(d, w_stride);
  if (rc) return rc;
  CK(cudaGetLastError());
  return WQL3D_OK;
}

int wql3d_interface_buffers(wql3d_domain *d, void **send, void **recv, int64_t *count, int32_t *elem_bytes) {
  if (!d || !d->has_iface || !d->iface.remote) return fail(WQL3D_EINVAL, "no remote interface side");
  if (send) *send = d->iface.send;
  if (recv) *recv = d->iface.recv;
  if (count) *count = (int64_t)9 * d->iface.ny * d->iface.nz;
  if (elem_bytes) *elem_bytes = d->fp32 ? 4 : 8;
  return WQL3D_OK;
}

int wql3d_pack_interface(wql3d_domain *d) {
  if (!d || !d->has_iface || !d->iface.remote) return fail(WQL3D_EINVAL, "no remote interface side");
  const int n = d->iface.ny * d->iface.nz;
  if (d->fp32) k_pack_face<float><<<(n + 127) / 128, 128, 0, d->stream>>>(d->bf[0], d->cur, d->iface.remote, (float *)d->iface.send);
  else k_pack_face<double><<<(n + 127) / 128, 128, 0, d->stream>>>(d->bd[0], d->cur, d->iface.remote, (double *)d->iface.send);
  d->launches++;
  CK(cudaGetLastError());
  return WQL3D_OK;
}

int wql3d_halo_buffers(wql3d_domain *d, int kind, void **send, void **recv, int64_t *count, int32_t *elem_bytes) {
  if (!d || !d->slab) return fail(WQL3D_EINVAL, "not an s-slab domain");
  if (kind != WQL3D_HALO_FIELDS && kind != WQL3D_HALO_METRIC) return fail(WQL3D_EINVAL, "halo kind");
  const int ncomp = kind == WQL3D_HALO_FIELDS ? 9 : 10;
  if (send) *send = d->halo_send;
  if (recv) *recv = d->halo_recv;
  if (count) *count = (int64_t)ncomp * 3 * d->hb[0].nq * d->hb[0].nr;
  if (elem_bytes) *elem_bytes = d->fp32 ? 4 : 8;
  return WQL3D_OK;
}

int wql3d_pack_halo(wql3d_domain *d, int kind) {
  if (!d || !d->slab) return fail(WQL3D_EINVAL, "not an s-slab domain");
  if (kind != WQL3D_HALO_FIELDS && kind != WQL3D_HALO_METRIC) return fail(WQL3D_EINVAL, "halo kind");
  return d->fp32 ? halo_launch<float>(d, d->bf[0], kind, 0) : halo_launch<double>(d, d->bd[0], kind, 0);
}

int wql3d_unpack_halo(wql3d_domain *d, int kind) {
  if (!d || !d->slab) return fail(WQL3D_EINVAL, "not an s-slab domain");
  if (kind != WQL3D_HALO_FIELDS && kind != WQL3D_HALO_METRIC) return fail(WQL3D_EINVAL, "halo kind");
  return d->fp32 ? halo_launch<float>(d, d->bf[0], kind, 1) : halo_launch<double>(d, d->bd[0], kind, 1);
}

int wql3d_get_interface_material(wql3d_domain *d, double *M) {
  if (!d || !d->has_iface || !d->iface.remote || !M) return fail(WQL3D_EINVAL, "no remote interface side");
  const int n = d->iface.ny * d->iface.nz;
  // the receive buffer is free between stages: stage the material through it
  if (d->fp32) {
    k_pack_face_material<float><<<(n + 127) / 128, 128, 0, d->stream>>>(d->bf[0], d->iface.remote, (float *)d->iface.recv);
    std::vector<float> h((size_t)3 * n);
    CK(cudaMemcpyAsync(h.data(), d->iface.recv, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, d->stream));
    CK(cudaStreamSynchronize(d->stream));
    for (size_t i = 0; i < h.size(); ++i) M[i] = h[i];
  } else {
    k_pack_face_material<double><<<(n + 127) / 128, 128, 0, d->stream>>>(d->bd[0], d->iface.remote, (double *)d->iface.recv);
    CK(cudaMemcpyAsync(M, d->iface.recv, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, d->stream));
    CK(cudaStreamSynchronize(d->stream));
  }
  return WQL3D_OK;
}

int wql3d_set_interface_remote_material(wql3d_domain *d, const double *M) {
  if (!d || !d->has_iface || !d->iface.remote || !M) return fail(WQL3D_EINVAL, "no remote interface side");
  const int n = d->iface.ny * d->iface.nz;
  if (d->fp32) {
    std::vector<float> h((size_t)3 * n);
    for (size_t i = 0; i < h.size(); ++i) h[i] = (float)M[i];
    CK(cudaMemcpyAsync(d->iface.oppM, h.data(), sizeof(float) * 3 * n, cudaMemcpyHostToDevice, d->stream));
    CK(cudaStreamSynchronize(d->stream));
  } else {
    CK(cudaMemcpyAsync(d->iface.oppM, M, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, d->stream));
    CK(cudaStreamSynchronize(d->stream));
  }
  return WQL3D_OK;
}

int wql3d_time_step(wql3d_domain *d, double dt, int n, int w_stride) {
  if (!d) return fail(WQL3D_EINVAL, "null domain");
  if (d->has_iface && d->iface.remote)
    return fail(WQL3D_ESTATE, "remote interface side: drive with wql3d_begin_step / pack / exchange / wql3d_stage");
  if (d->slab)
    return fail(WQL3D_ESTATE, "s-slab domain: drive with wql3d_begin_step / halo pack / exchange / unpack / wql3d_stage");
  DevTime h;
  CK(cudaMemcpyAsync(&h, d->time, sizeof(h), cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  h.n = n;
  CK(cudaMemcpyAsync(d->time, &h, sizeof(h), cudaMemcpyHostToDevice, d->stream));
  int rc = d->fp32 ? enqueue_step<float>(d, dt, w_stride) : enqueue_step<double>(d, dt, w_stride);
  if (rc) return rc;
  CK(cudaGetLastError());
  return WQL3D_OK;
}

int wql3d_run(wql3d_domain *d, double dt, int n_first, int nsteps, int w_stride) {
  if (!d) return fail(WQL3D_EINVAL, "null domain");
  if (d->has_iface && d->iface.remote)
    return fail(WQL3D_ESTATE, "remote interface side: drive with wql3d_begin_step / pack / exchange / wql3d_stage");
  if (d->slab)
    return fail(WQL3D_ESTATE, "s-slab domain: drive with wql3d_begin_step / halo pack / exchange / unpack / wql3d_stage");
  if (nsteps < 0) return fail(WQL3D_EINVAL, "nsteps");
  DevTime h;
  CK(cudaMemcpyAsync(&h, d->time, sizeof(h), cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  h.n = n_first;
  CK(cudaMemcpyAsync(d->time, &h, sizeof(h), cudaMemcpyHostToDevice, d->stream));
  return d->fp32 ? run_steps<float>(d, dt, nsteps, w_stride) : run_steps<double>(d, dt, nsteps, w_stride);
}

int wql3d_scale_rates(wql3d_domain *d, double A) {
  if (!d) return fail(WQL3D_EINVAL, "null domain");
  // A*DF and the point-local memory-variable / PML rates, whole arrays
  for (int i = 0; i < d->nblocks; ++i) {
    if (d->fp32) {
      Blk<float> &b = d->bf[i];
      k_scale_T<float><<<1184, 256, 0, d->stream>>>(b.DF, 9 * b.vol, A);
      if (b.nmech) k_scale_T<float><<<1184, 256, 0, d->stream>>>(b.deta, (long long)6 * b.nmech * b.vol, A);
      for (int f = 0; f < 6; ++f)
        if (b.pml_on[f]) k_scale_T<float><<<1184, 256, 0, d->stream>>>(b.DQ[f], 9 * b.pvol[f], A);
    } else {
      Blk<double> &b = d->bd[i];
      k_scale_T<double><<<1184, 256, 0, d->stream>>>(b.DF, 9 * b.vol, A);
      if (b.nmech) k_scale_T<double><<<1184, 256, 0, d->stream>>>(b.deta, (long long)6 * b.nmech * b.vol, A);
      for (int f = 0; f < 6; ++f)
        if (b.pml_on[f]) k_scale_T<double><<<1184, 256, 0, d->stream>>>(b.DQ[f], 9 * b.pvol[f], A);
    }
    d->launches++;
  }
  if (d->has_iface) {
    iface_scale(d->iface, A, d->stream);
    d->launches++;
  }
  CK(cudaGetLastError());
  return WQL3D_OK;
}

int wql3d_set_rates_rhs(wql3d_domain *d) {
  if (!d) return fail(WQL3D_EINVAL, "null domain");
  // stage index 1 makes the source evaluate at the current domain time
  StageArgs a;
  a.cur = d->cur;
  a.flags = F_RHS | F_SOURCE;
  a.stage = 1;
  a.A = 1.0;
  a.Bdt = 0.0;
  a.dt = 0.0;
  a.time = d->time;
  for (int i = 0; i < d->nblocks; ++i) {
    if (d->fp32) launch_stage<float>(d, i, a);
    else launch_stage<double>(d, i, a);
  }
  CK(cudaGetLastError());
  return WQL3D_OK;
}

int wql3d_try_traditional_rhs(wql3d_domain *d, int *handled) {
  if (handled) *handled = 0;
  int rc = wql3d_set_rates_rhs(d);
  if (rc) return rc;
  if (handled) *handled = 1;
  return WQL3D_OK;
}

int wql3d_enforce_bound_iface_conditions(wql3d_domain *d, int stage) {
  if (!d) return fail(WQL3D_EINVAL, "null domain");
  StageArgs a;
  a.cur = d->cur;
  a.flags = F_SAT | (d->has_iface ? F_ISAT : 0);
  a.stage = stage < 1 ? 1 : stage;
  a.A = 1.0;
  a.Bdt = 0.0;
  a.dt = 0.0;
  a.time = d->time;
  if (d->has_iface) {
    if (d->fp32) launch_iface<float>(d->iface, d->bf[0], d->bf[1], a, d->stream);
    else launch_iface<double>(d->iface, d->bd[0], d->bd[1], a, d->stream);
    d->launches++;
  }
  for (int i = 0; i < d->nblocks; ++i) {
    if (d->fp32) launch_stage<float>(d, i, a);
    else launch_stage<double>(d, i, a);
  }
  CK(cudaGetLastError());
  return WQL3D_OK;
}

int wql3d_update_fields(wql3d_domain *d, double dt) {
  if (!d) return fail(WQL3D_EINVAL, "null domain");
  for (int i = 0; i < d->nblocks; ++i) {
    if (d->fp32) {
      Blk<float> &b = d->bf[i];
      dim3 th(32, 4, 2), gr((b.nx + 31) / 32, (b.ny + 3) / 4, (b.nz + 1) / 2);
      k_update_inplace<float><<<gr, th, 0, d->stream>>>(b, d->cur, dt);
      if (b.nmech) k_axpy_T<float><<<1184, 256, 0, d->stream>>>(b.eta, b.deta, (long long)6 * b.nmech * b.vol, dt);
      for (int f = 0; f < 6; ++f)
        if (b.pml_on[f]) k_axpy_T<float><<<1184, 256, 0, d->stream>>>(b.Q[f], b.DQ[f], 9 * b.pvol[f], dt);
    } else {
      Blk<double> &b = d->bd[i];
      dim3 th(32, 4, 2), gr((b.nx + 31) / 32, (b.ny + 3) / 4, (b.nz + 1) / 2);
      k_update_inplace<double><<<gr, th, 0, d->stream>>>(b, d->cur, dt);
      if (b.nmech) k_axpy_T<double><<<1184, 256, 0, d->stream>>>(b.eta, b.deta, (long long)6 * b.nmech * b.vol, dt);
      for (int f = 0; f < 6; ++f)
        if (b.pml_on[f]) k_axpy_T<double><<<1184, 256, 0, d->stream>>>(b.Q[f], b.DQ[f], 9 * b.pvol[f], dt);
    }
    d->launches++;
  }
  if (d->has_iface) {
    if (d->fp32) launch_iface_update<float>(d->iface, d->bf[0], d->bf[1], dt, d->stream);
    else launch_iface_update<double>(d->iface, d->bd[0], d->bd[1], dt, d->stream);
    d->launches++;
  }
  CK(cudaGetLastError());
  return WQL3D_OK;
}

int wql3d_scale_rate_array(double *rate, int64_t n, double coefficient, void *stream) {
  if (n < 0 || (n > 0 && !rate)) return fail(WQL3D_EINVAL, "rate array");
  if (n == 0) return WQL3D_OK;
  int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
  k_scale_array<<<blocks, 256, 0, (cudaStream_t)stream>>>(rate, n, coefficient);
  CK(cudaGetLastError());
  return WQL3D_OK;
}

int wql3d_update_state_array(double *state, const double *rate, int64_t n, double increment, void *stream) {
  if (n < 0 || (n > 0 && (!state || !rate))) return fail(WQL3D_EINVAL, "state/rate array");
  if (n == 0) return WQL3D_OK;
  int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
  k_axpy_array<<<blocks, 256, 0, (cudaStream_t)stream>>>(state, rate, n, increment);
  CK(cudaGetLastError());
  return WQL3D_OK;
}

int wql3d_traditional_cartesian_rhs(const double *field, double *rate, const double *metricx, const double *metricy,
                                    const double *metricz, const double *material, int32_t n1, int32_t n2, int32_t n3,
                                    int32_t nm, int32_t nmat, int32_t xlo, int32_t xhi, int32_t ylo, int32_t yhi,
                                    int32_t zlo, int32_t zhi, double hq, double hr, double hs, void *stream) {
  if (!field || !rate || !metricx || !metricy || !metricz || !material) return fail(WQL3D_EINVAL, "rhs arrays");
  if (n1 < 1 || n2 < 1 || n3 < 1 || nm < 3 || nmat < 3) return fail(WQL3D_EINVAL, "rhs array shape");
  // the box must leave the three stencil points on each side inside the arrays
  if (xlo < 4 || xhi > n1 - 3 || ylo < 4 || yhi > n2 - 3 || zlo < 4 || zhi > n3 - 3)
    return fail(WQL3D_EINVAL, "rhs interior bounds");
  if (xlo > xhi || ylo > yhi || zlo > zhi) return WQL3D_OK;
  CartRhsArgs a;
  a.field = field; a.rate = rate; a.mx = metricx; a.my = metricy; a.mz = metricz; a.mat = material;
  a.n1 = n1; a.n2 = n2; a.n3 = n3;
  a.lo[0] = xlo; a.lo[1] = ylo; a.lo[2] = zlo;
  a.ext[0] = xhi - xlo + 1; a.ext[1] = yhi - ylo + 1; a.ext[2] = zhi - zlo + 1;
  const double c[3] = {0.75, -0.15, 1.0 / 60.0};
  for (int s = 0; s < 3; ++s) {
    a.cx[s] = c[s] / hq;
    a.cy[s] = c[s] / hr;
    a.cz[s] = c[s] / hs;
  }
  const long long npts = (long long)a.ext[0] * a.ext[1] * a.ext[2];
  const unsigned g = (unsigned)std::min<long long>((npts + 255) / 256, 148LL * 64);
  k_trad_cart_rhs<<<g, 256, 0, (cudaStream_t)stream>>>(a);
  CK(cudaGetLastError());
  return WQL3D_OK;
}

int wql3d_get_seismograms(wql3d_domain *d, int bi, double *out, int32_t *nsamples) {
  DOM_CHECK(d, bi);
  DevTime h;
  CK(cudaMemcpyAsync(&h, d->time, sizeof(h), cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  int ns = std::min(h.nsamp, d->desc.max_samples);
  if (nsamples) *nsamples = ns;
  int nrec = d->hb[bi].nrec;
  if (out && ns > 0 && nrec > 0) {
    const double *src = d->fp32 ? d->bf[bi].seis : d->bd[bi].seis;
    CK(cudaMemcpyAsync(out, src, sizeof(double) * (size_t)ns * nrec * 4, cudaMemcpyDeviceToHost, d->stream));
    CK(cudaStreamSynchronize(d->stream));
  }
  return WQL3D_OK;
}

int wql3d_receiver_index(wql3d_domain *d, int bi, int32_t *idx) {
  DOM_CHECK(d, bi);
  if (d->hb[bi].nrec > 0) memcpy(idx, d->hb[bi].ridx.data(), sizeof(int32_t) * 3 * d->hb[bi].nrec);
  return WQL3D_OK;
}

int wql3d_final_state(wql3d_domain *d, double *max_field, double *max_memory, double *block_max) {
  if (!d) return fail(WQL3D_EINVAL, "null domain");
  return d->fp32 ? final_state<float>(d, max_field, max_memory, block_max)
                 : final_state<double>(d, max_field, max_memory, block_max);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Discrete adjoint (no counterpart in the reference)
// ---------------------------------------------------------------------------
namespace {

// transposed derivative rows of the traditional-6 operator for an axis of n
// points: row q lists (p - q, D[p][q]) over the rows p that read point q,
// with the forward's row choice (left closure for p <= 6, right closure for
// p >= n - 5, central row otherwise)
void transposed_rows(int n, int lit, std::vector<int> &off, std::vector<double> &c) {
  std::vector<double> D((size_t)n * n, 0.0);
  for (int p = 1; p <= n; ++p) {
    if (p <= 6) {
      const int r = p - 1;
      for (int k = 0; k < kSbpCnt[r]; ++k) D[(size_t)(p - 1) * n + (kSbpIdx[r][k] - 1)] += kSbpC[lit][r][k];
    } else if (p >= n - 5) {
      const int r = n - p;
      for (int k = 0; k < kSbpCnt[r]; ++k) D[(size_t)(p - 1) * n + (n - kSbpIdx[r][k])] += -kSbpC[lit][r][k];
    } else {
      const double cc[6] = {-1.0 / 60.0, 0.15, -0.75, 0.75, -0.15, 1.0 / 60.0};
      const int oo[6] = {-3, -2, -1, 1, 2, 3};
      for (int k = 0; k < 6; ++k) D[(size_t)(p - 1) * n + (p - 1 + oo[k])] += cc[k];
    }
  }
  off.assign((size_t)n * ADJ_TW, 0);
  c.assign((size_t)n * ADJ_TW, 0.0);
  for (int q = 1; q <= n; ++q) {
    int k = 0;
    for (int p = 1; p <= n; ++p) {
      const double v = D[(size_t)(p - 1) * n + (q - 1)];
      if (v == 0.0) continue;
      off[(size_t)(q - 1) * ADJ_TW + k] = p - q;
      c[(size_t)(q - 1) * ADJ_TW + k] = v;
      ++k;
    }
  }
}

// recorded steps carry the stage inputs' derivative terms when the block's
// stages run the fused curvilinear kernel (the Cartesian kernels do not write
// them; the adjoint then recomputes them)
bool record_terms(wql3d_domain *d) {
  return d->hb[0].mesh == WQL3D_MESH_CURVILINEAR && !tuning().generic && curv_stage_fused(d->bd[0]);
}

int adjoint_supported(wql3d_domain *d) {
  if (d->fp32 || d->nblocks != 1 || d->response != WQL3D_ELASTIC || d->slab || d->desc.remote_side || d->desc.mms)
    return fail(WQL3D_EINVAL, "the adjoint covers one FP64 elastic block (no interface, slab or MMS)");
  const wql3d_block_desc &bd = d->desc.block[0];
  for (int f = 0; f < 6; ++f)
    if (bd.pml[f] && bd.npml > 0) return fail(WQL3D_EINVAL, "the adjoint covers blocks without PML");
  if (bd.fd_operator != WQL3D_FD_TRADITIONAL6) return fail(WQL3D_EINVAL, "the adjoint covers traditional-6");
  if (bd.nq < 13 || bd.nr < 13 || bd.ns < 13) return fail(WQL3D_EINVAL, "the adjoint needs 13 points per axis");
  return WQL3D_OK;
}

}  // namespace

extern "C" {

int wql3d_adjoint_enable(wql3d_domain *d) {
  if (!d) return fail(WQL3D_EINVAL, "null domain");
  if (d->adj_on) return WQL3D_OK;
  if (int rc = adjoint_supported(d)) return rc;
  Blk<double> &b = d->bd[0];
  const size_t V = (size_t)b.vol;
  AdjBlk &A = d->adj;
  Alloc &M = d->mem;
  CK(M.get(&A.Fb, 9 * V));
  CK(M.get(&A.DFb, 9 * V));
  CK(M.get(&A.R, 9 * V));
  CK(M.get(&A.ZY, 12 * V));
  CK(M.get(&A.g, 3 * V));
  CK(M.get(&A.gM, (size_t)6 * std::max(1, b.nsrc)));
  for (int s = 0; s < 5; ++s) CK(M.get(&A.S[s], 9 * V, false));
  CK(M.get(&d->adj_res, (size_t)3 * std::max(1, b.nrec)));
  const int nn[3] = {b.nx, b.ny, b.nz};
  for (int a = 0; a < 3; ++a) {
    std::vector<int> off;
    std::vector<double> c;
    transposed_rows(nn[a], b.lit, off, c);
    int *doff;
    double *dc;
    CK(M.get(&doff, off.size()));
    CK(M.get(&dc, c.size()));
    CK(cudaMemcpyAsync(doff, off.data(), sizeof(int) * off.size(), cudaMemcpyHostToDevice, d->stream));
    CK(cudaMemcpyAsync(dc, c.data(), sizeof(double) * c.size(), cudaMemcpyHostToDevice, d->stream));
    A.toff[a] = doff;
    A.tc[a] = dc;
  }
  A.res = d->adj_res;
  CK(cudaStreamSynchronize(d->stream));
  d->adj_on = true;
  return WQL3D_OK;
}

int wql3d_adjoint_reset(wql3d_domain *d) {
  if (!d || !d->adj_on) return fail(WQL3D_ESTATE, "adjoint not enabled");
  const size_t V = (size_t)d->bd[0].vol;
  AdjBlk &A = d->adj;
  CK(cudaMemsetAsync(A.Fb, 0, sizeof(double) * 9 * V, d->stream));
  CK(cudaMemsetAsync(A.DFb, 0, sizeof(double) * 9 * V, d->stream));
  CK(cudaMemsetAsync(A.g, 0, sizeof(double) * 3 * V, d->stream));
  CK(cudaMemsetAsync(A.gM, 0, sizeof(double) * 6 * std::max(1, d->bd[0].nsrc), d->stream));
  CK(cudaStreamSynchronize(d->stream));
  return WQL3D_OK;
}

int wql3d_adjoint_step(wql3d_domain *d, int n, double dt) {
  if (!d || !d->adj_on) return fail(WQL3D_ESTATE, "adjoint not enabled");
  Blk<double> &b = d->bd[0];
  AdjBlk &A = d->adj;
  const size_t bytes = sizeof(double) * 9 * (size_t)b.vol;
  DevTime h;
  CK(cudaMemcpyAsync(&h, d->time, sizeof(h), cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  const double t0 = h.t;
  (void)n;
  // stage inputs F^(0..4) of this step, recomputed from the current fields
  const int cur0 = d->cur;
  CK(cudaMemcpyAsync(A.S[0], d->cur ? b.F1 : b.F0, bytes, cudaMemcpyDeviceToDevice, d->stream));
  for (int s = 1; s <= 4; ++s) {
    if (int rc = enqueue_stage<double>(d, s, dt, F_ALL)) return rc;
    CK(cudaMemcpyAsync(A.S[s], d->cur ? b.F1 : b.F0, bytes, cudaMemcpyDeviceToDevice, d->stream));
  }
  // leave the domain's fields at F^(0) = F_n
  d->cur = cur0;
  CK(cudaMemcpyAsync(d->cur ? b.F1 : b.F0, A.S[0], bytes, cudaMemcpyDeviceToDevice, d->stream));
  // reversed stages 5..1
  for (int s = 5; s >= 1; --s) {
    adj_launch_stage(b, A, s, kRkB[s - 1] * dt, kRkA[s - 1], d->stream, &d->launches);
    adj_launch_moment(b, A, t0 + kRkC[s - 1] * dt, d->stream, &d->launches);
  }
  CK(cudaGetLastError());
  return WQL3D_OK;
}

int wql3d_record_step(wql3d_domain *d, double dt, int n, int w_stride, double *dev_out) {
  if (!d || d->fp32 || d->nblocks != 1 || d->slab || (d->has_iface && d->iface.remote) || !dev_out)
    return fail(WQL3D_EINVAL, "recording covers one-block FP64 domains and a device buffer");
  Blk<double> &b = d->bd[0];
  const size_t ne = (size_t)9 * b.vol;
  DevTime h;
  CK(cudaMemcpyAsync(&h, d->time, sizeof(h), cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  h.n = n;
  CK(cudaMemcpyAsync(d->time, &h, sizeof(h), cudaMemcpyHostToDevice, d->stream));
  if (int rc = enqueue_sample<double>(d, w_stride)) return rc;
  // stage inputs, then (blocks on the fused curvilinear kernel) the stage
  // inputs' derivative terms written by the stage kernel itself
  const bool terms = record_terms(d);
  for (int s = 1; s <= 5; ++s) {
    CK(cudaMemcpyAsync(dev_out + (s - 1) * ne, d->cur ? b.F1 : b.F0, sizeof(double) * ne, cudaMemcpyDeviceToDevice,
                       d->stream));
    if (int rc = enqueue_stage<double>(d, s, dt, F_ALL, terms ? (void *)(dev_out + (4 + s) * ne) : nullptr)) return rc;
  }
  k_advance<<<1, 32, 0, d->stream>>>(d->time, dt);
  d->launches++;
  CK(cudaGetLastError());
  return WQL3D_OK;
}

int wql3d_adjoint_step_recorded(wql3d_domain *d, int n, double dt, double t_n, const double *dev_in) {
  if (!d || !d->adj_on) return fail(WQL3D_ESTATE, "adjoint not enabled");
  if (!dev_in) return fail(WQL3D_EINVAL, "null stage inputs");
  (void)n;
  Blk<double> &b = d->bd[0];
  AdjBlk A = d->adj;
  const size_t ne = (size_t)9 * b.vol;
  const bool terms = record_terms(d);
  for (int s = 0; s < 5; ++s) {
    A.S[s] = const_cast<double *>(dev_in) + s * ne;
    A.E[s] = terms ? dev_in + (5 + s) * ne : nullptr;
  }
  for (int s = 5; s >= 1; --s) {
    adj_launch_stage(b, A, s, kRkB[s - 1] * dt, kRkA[s - 1], d->stream, &d->launches);
    adj_launch_moment(b, A, t_n + kRkC[s - 1] * dt, d->stream, &d->launches);
  }
  CK(cudaGetLastError());
  return WQL3D_OK;
}

int wql3d_adjoint_add_receivers(wql3d_domain *d, int bi, const double *res) {
  if (!d || !d->adj_on) return fail(WQL3D_ESTATE, "adjoint not enabled");
  if (bi != 0 || !res) return fail(WQL3D_EINVAL, "block / residuals");
  const int nrec = d->bd[0].nrec;
  if (nrec <= 0) return WQL3D_OK;
  CK(cudaMemcpyAsync(d->adj_res, res, sizeof(double) * 3 * nrec, cudaMemcpyHostToDevice, d->stream));
  adj_launch_receivers(d->bd[0], d->adj, d->stream, &d->launches);
  CK(cudaStreamSynchronize(d->stream));
  return WQL3D_OK;
}

int wql3d_adjoint_rhs(wql3d_domain *d, int bi, const double *R, double *Fbar, double *g) {
  if (!d || !d->adj_on) return fail(WQL3D_ESTATE, "adjoint not enabled");
  if (bi != 0 || !R || !Fbar || !g) return fail(WQL3D_EINVAL, "arguments");
  Blk<double> &b = d->bd[0];
  AdjBlk &A = d->adj;
  const size_t V = (size_t)b.vol;
  CK(cudaMemsetAsync(A.Fb, 0, sizeof(double) * 9 * V, d->stream));
  CK(cudaMemsetAsync(A.g, 0, sizeof(double) * 3 * V, d->stream));
  if (int rc = put_array<double>(d, d->hb[0], A.DFb, 9, R, 0)) return rc;
  CK(cudaMemcpyAsync(A.S[0], d->cur ? b.F1 : b.F0, sizeof(double) * 9 * V, cudaMemcpyDeviceToDevice, d->stream));
  adj_launch_stage(b, A, 1, 0.0, 0.0, d->stream, &d->launches);
  CK(cudaGetLastError());
  if (int rc = get_array<double>(d, d->hb[0], A.Fb, 9, Fbar, 0)) return rc;
  return get_array<double>(d, d->hb[0], A.g, 3, g, 0);
}

int wql3d_get_adjoint_fields(wql3d_domain *d, int bi, double *Fbar) {
  if (!d || !d->adj_on) return fail(WQL3D_ESTATE, "adjoint not enabled");
  if (bi != 0 || !Fbar) return fail(WQL3D_EINVAL, "arguments");
  return get_array<double>(d, d->hb[0], d->adj.Fb, 9, Fbar, 0);
}

int wql3d_get_adjoint_gradient(wql3d_domain *d, int bi, double *g_material, double *g_moment) {
  if (!d || !d->adj_on) return fail(WQL3D_ESTATE, "adjoint not enabled");
  if (bi != 0) return fail(WQL3D_EINVAL, "block");
  if (g_material)
    if (int rc = get_array<double>(d, d->hb[0], d->adj.g, 3, g_material, 0)) return rc;
  if (g_moment && d->bd[0].nsrc > 0) {
    CK(cudaMemcpyAsync(g_moment, d->adj.gM, sizeof(double) * 6 * d->bd[0].nsrc, cudaMemcpyDeviceToHost, d->stream));
    CK(cudaStreamSynchronize(d->stream));
  }
  return WQL3D_OK;
}

int wql3d_store_fields(wql3d_domain *d, int bi, double *dev_dst) {
  DOM_CHECK(d, bi);
  if (d->fp32 || !dev_dst) return fail(WQL3D_EINVAL, "FP64 domain and a device array");
  const Blk<double> &b = d->bd[bi];
  CK(cudaMemcpyAsync(dev_dst, d->cur ? b.F1 : b.F0, sizeof(double) * 9 * (size_t)b.vol, cudaMemcpyDeviceToDevice,
                     d->stream));
  return WQL3D_OK;
}

int wql3d_load_fields(wql3d_domain *d, int bi, const double *dev_src) {
  DOM_CHECK(d, bi);
  if (d->fp32 || !dev_src) return fail(WQL3D_EINVAL, "FP64 domain and a device array");
  const Blk<double> &b = d->bd[bi];
  CK(cudaMemcpyAsync(d->cur ? b.F1 : b.F0, dev_src, sizeof(double) * 9 * (size_t)b.vol, cudaMemcpyDeviceToDevice,
                     d->stream));
  return WQL3D_OK;
}

int wql3d_field_volume(wql3d_domain *d, int bi, int64_t *elements) {
  DOM_CHECK(d, bi);
  if (!elements) return fail(WQL3D_EINVAL, "null argument");
  *elements = (int64_t)9 * (d->fp32 ? d->bf[bi].vol : d->bd[bi].vol);
  return WQL3D_OK;
}

int wql3d_get_plane(wql3d_domain *d, int bi, int axis, int index, int c0, int ncomp, double *out) {
  DOM_CHECK(d, bi);
  const HostBlock &h = d->hb[bi];
  const int n[3] = {h.nq, h.nr, h.ns};
  if (!out || axis < 1 || axis > 3 || index < 1 || index > n[axis - 1] || c0 < 0 || ncomp < 1 || c0 + ncomp > 9)
    return fail(WQL3D_EINVAL, "plane");
  const int dir = axis - 1;
  const long long total = (long long)(dir == 0 ? h.nr : h.nq) * (dir == 2 ? h.nr : h.ns) * ncomp;
  if (total > d->plane_cap) return fail(WQL3D_EINVAL, "plane");
  const unsigned g = (unsigned)std::min<long long>((total + 255) / 256, 4096);
  if (d->fp32)
    k_plane_gather<float><<<g, 256, 0, d->stream>>>(d->bf[bi], d->cur ? d->bf[bi].F1 : d->bf[bi].F0, dir, index, c0,
                                                    ncomp, d->plane);
  else
    k_plane_gather<double><<<g, 256, 0, d->stream>>>(d->bd[bi], d->cur ? d->bd[bi].F1 : d->bd[bi].F0, dir, index, c0,
                                                     ncomp, d->plane);
  ++d->launches;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, d->plane, sizeof(double) * total, cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  return WQL3D_OK;
}

int wql3d_check_status(wql3d_domain *d, int32_t *bad_step) {
  if (!d) return fail(WQL3D_EINVAL, "null domain");
  DevTime h;
  CK(cudaMemcpyAsync(&h, d->time, sizeof(h), cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  CK(cudaGetLastError());
  if (bad_step) *bad_step = h.bad;
  if (h.stall) return fail(WQL3D_ECUDA, "a bounded wait in a stage kernel gave up: the fields are void");
  if (h.bad) return fail(WQL3D_ENONFINITE, "non-finite station value at step " + std::to_string(h.bad) +
                                                " (RUN-STATION-001)");
  return WQL3D_OK;
}

int wql3d_reset_samples(wql3d_domain *d) {
  if (!d) return fail(WQL3D_EINVAL, "null domain");
  DevTime h;
  CK(cudaMemcpyAsync(&h, d->time, sizeof(h), cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  h.nsamp = 0;
  CK(cudaMemcpyAsync(d->time, &h, sizeof(h), cudaMemcpyHostToDevice, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  return WQL3D_OK;
}

int wql3d_set_material(wql3d_domain *d, int bi, const double *M) {
  DOM_CHECK(d, bi);
  if (!M) return fail(WQL3D_EINVAL, "null material");
  return d->fp32 ? put_array<float>(d, d->hb[bi], d->bf[bi].M, 3, M, 0)
                 : put_array<double>(d, d->hb[bi], d->bd[bi].M, 3, M, 0);
}

int wql3d_set_moment(wql3d_domain *d, int bi, const double *m6) {
  DOM_CHECK(d, bi);
  const int ns = d->fp32 ? d->bf[bi].nsrc : d->bd[bi].nsrc;
  if (ns <= 0) return WQL3D_OK;
  if (!m6) return fail(WQL3D_EINVAL, "null moment");
  DevSource *ds = const_cast<DevSource *>(d->fp32 ? d->bf[bi].src : d->bd[bi].src);
  std::vector<DevSource> hs((size_t)ns);
  CK(cudaMemcpyAsync(hs.data(), ds, sizeof(DevSource) * ns, cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  for (int i = 0; i < ns; ++i)
    for (int c = 0; c < 6; ++c) hs[(size_t)i].par[2 + c] = m6[6 * i + c];
  CK(cudaMemcpyAsync(ds, hs.data(), sizeof(DevSource) * ns, cudaMemcpyHostToDevice, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  return WQL3D_OK;
}

}  // extern "C"

extern "C" {

// ---------------------------------------------------------------------------
// Batched independent shots (no counterpart in the reference)
// ---------------------------------------------------------------------------
}  // extern "C"

struct wql3d_batch {
  int n = 0;
  int fp32 = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev = nullptr;
  cudaStream_t side = nullptr;               // the shells' stream (fork / join per stage)
  cudaEvent_t fork = nullptr, join = nullptr;
  std::vector<wql3d_domain *> doms;
  Alloc mem;
  void *blks = nullptr;           // device array of Blk<T>
  DevTime **times = nullptr;      // device array of the shots' DevTime pointers
  struct Cls {
    int resp = 0, sep = 0;
    std::vector<int> shots;
    int *d_shots = nullptr, *d_tile = nullptr, *d_shell = nullptr;
    int tiles = 0, shell_ctas = 0;
  } cls[8];
  int zchunk = 12;
  int tuned = 0;
  int cur = 0;
  cudaGraphExec_t graph = nullptr;
  double g_dt = 0.0;
  int g_w = -1, g_cur = -1, g_z = -1;
  int64_t g_launches = 0, launches = 0;
  std::vector<std::pair<int, float>> tune_log;   // (zchunk, ms per step) of the tuning steps
};

namespace {

// the classes' interior tile prefix sums for the current zchunk
int batch_tiles(wql3d_batch *bt) {
  for (auto &c : bt->cls) {
    if (c.shots.empty()) continue;
    std::vector<int> pre(c.shots.size() + 1, 0);
    for (size_t i = 0; i < c.shots.size(); ++i) {
      const wql3d_domain *d = bt->doms[(size_t)c.shots[i]];
      const int *lo = bt->fp32 ? d->bf[0].lo : d->bd[0].lo, *hi = bt->fp32 ? d->bf[0].hi : d->bd[0].hi;
      const int nxi = hi[0] - lo[0] + 1, nyi = hi[1] - lo[1] + 1, nzi = hi[2] - lo[2] + 1;
      const int t = (nxi > 0 && nyi > 0 && nzi > 0)
                        ? ((nxi + 31) / 32) * ((nyi + 3) / 4) * ((nzi + bt->zchunk - 1) / bt->zchunk) : 0;
      pre[i + 1] = pre[i] + t;
    }
    c.tiles = pre.back();
    CK(cudaMemcpyAsync(c.d_tile, pre.data(), sizeof(int) * pre.size(), cudaMemcpyHostToDevice, bt->stream));
    CK(cudaStreamSynchronize(bt->stream));
  }
  return WQL3D_OK;
}

template <typename T>
void batch_enqueue_step(wql3d_batch *bt, double dt, int w_stride) {
  launch_batch_sample<T>((const Blk<T> *)bt->blks, bt->times, bt->n, bt->cur, w_stride, bt->stream, &bt->launches);
  BatchClass<T> cl[8];
  int ncl = 0;
  for (auto &c : bt->cls) {
    if (c.shots.empty()) continue;
    BatchClass<T> &b = cl[ncl++];
    b.resp = c.resp;
    b.sep = c.sep;
    b.nshots = (int)c.shots.size();
    b.shots = c.d_shots;
    b.tile_prefix = c.d_tile;
    b.shell_prefix = c.d_shell;
    b.tiles = c.tiles;
    b.shell_ctas = c.shell_ctas;
    b.blks = (const Blk<T> *)bt->blks;
    b.times = bt->times;
  }
  for (int st = 1; st <= 5; ++st) {
    StageArgs a;
    a.cur = bt->cur;
    a.flags = F_ALL;
    a.stage = st;
    a.A = kRkA[st - 1];
    a.Bdt = kRkB[st - 1] * dt;
    a.dt = dt;
    a.time = nullptr;
    launch_batch_stage<T>(cl, ncl, a, bt->zchunk, bt->stream, tuning().overlap ? bt->side : nullptr, bt->fork,
                          bt->join, &bt->launches);
    bt->cur ^= 1;
  }
  launch_batch_advance<T>(bt->times, bt->n, dt, bt->stream, &bt->launches);
}

template <typename T>
int batch_run(wql3d_batch *bt, double dt, int nsteps, int w_stride) {
  // project-written tile autotuner: the first steps of the first run each try
  // one z-chunk length of the interior tiles (the arithmetic of a point does
  // not depend on it), timed with events; the fastest is kept
  if (!bt->tuned) {
    const int cand[6] = {4, 8, 12, 16, 24, 32};
    float best = 1e30f;
    int bestz = bt->zchunk;
    for (int i = 0; i < 6 && nsteps > 0; ++i) {
      bt->zchunk = cand[i];
      if (int rc = batch_tiles(bt)) return rc;
      cudaEvent_t e0, e1;
      CK(cudaEventCreate(&e0));
      CK(cudaEventCreate(&e1));
      CK(cudaEventRecord(e0, bt->stream));
      batch_enqueue_step<T>(bt, dt, w_stride);
      CK(cudaEventRecord(e1, bt->stream));
      CK(cudaEventSynchronize(e1));
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, e0, e1));
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      bt->tune_log.push_back({cand[i], ms});
      if (ms < best) { best = ms; bestz = cand[i]; }
      --nsteps;
    }
    bt->zchunk = bestz;
    if (int rc = batch_tiles(bt)) return rc;
    bt->tuned = 1;
  }
  // CUDA graph of two steps of the whole batch, replayed
  const int pairs = nsteps / 2;
  if (pairs > 0) {
    if (!bt->graph || bt->g_dt != dt || bt->g_w != w_stride || bt->g_cur != bt->cur || bt->g_z != bt->zchunk) {
      if (bt->graph) { cudaGraphExecDestroy(bt->graph); bt->graph = nullptr; }
      const int cur0 = bt->cur;
      const int64_t l0 = bt->launches;
      cudaGraph_t g;
      CK(cudaStreamBeginCapture(bt->stream, cudaStreamCaptureModeThreadLocal));
      batch_enqueue_step<T>(bt, dt, w_stride);
      batch_enqueue_step<T>(bt, dt, w_stride);
      CK(cudaStreamEndCapture(bt->stream, &g));
      CK(cudaGraphInstantiate(&bt->graph, g, 0));
      cudaGraphDestroy(g);
      bt->cur = cur0;
      bt->g_dt = dt;
      bt->g_w = w_stride;
      bt->g_cur = cur0;
      bt->g_z = bt->zchunk;
      bt->g_launches = bt->launches - l0;
      bt->launches = l0;
    }
    for (int k = 0; k < pairs; ++k) {
      CK(cudaGraphLaunch(bt->graph, bt->stream));
      bt->launches += bt->g_launches;
    }
  }
  if (nsteps % 2) batch_enqueue_step<T>(bt, dt, w_stride);
  CK(cudaGetLastError());
  return WQL3D_OK;
}

}  // namespace

extern "C" {

int wql3d_batch_create(wql3d_domain *const *domains, int32_t n, wql3d_batch **out) {
  if (!domains || n <= 0 || !out) return fail(WQL3D_EINVAL, "null argument");
  if (!domains[0]) return fail(WQL3D_EINVAL, "null domain");
  const int fp32 = domains[0]->fp32;
  for (int i = 0; i < n; ++i) {
    const wql3d_domain *d = domains[i];
    if (!d) return fail(WQL3D_EINVAL, "null domain");
    if (d->nblocks != 1 || d->slab || d->desc.remote_side || d->desc.mms || d->hb[0].mesh != WQL3D_MESH_CARTESIAN ||
        d->desc.block[0].fd_operator != WQL3D_FD_TRADITIONAL6 || d->fp32 != fp32 || d->cur != domains[0]->cur)
      return fail(WQL3D_EINVAL, "a batch holds one-block Cartesian traditional-6 domains of one precision");
    for (int f = 0; f < 6; ++f)
      if (d->desc.block[0].pml[f] && d->desc.block[0].npml > 0)
        return fail(WQL3D_EINVAL, "batched shots carry no PML");
  }
  wql3d_batch *bt = new wql3d_batch();
  bt->n = n;
  bt->fp32 = fp32;
  bt->doms.assign(domains, domains + n);
  bt->cur = domains[0]->cur;
  auto drop = [](wql3d_batch *b) {
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->join) cudaEventDestroy(b->join);
    if (b->side) cudaStreamDestroy(b->side);
    if (b->ev) cudaEventDestroy(b->ev);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
  };
  if (cudaStreamCreateWithFlags(&bt->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&bt->ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaStreamCreateWithFlags(&bt->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&bt->fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&bt->join, cudaEventDisableTiming) != cudaSuccess) {
    drop(bt);
    return fail(WQL3D_ECUDA, "batch stream");
  }
  bt->mem.stream = bt->stream;
  auto bad = [&](int code) {
    cudaStreamSynchronize(bt->stream);
    bt->mem.release();
    drop(bt);
    return code;
  };
  const size_t bsz = fp32 ? sizeof(Blk<float>) : sizeof(Blk<double>);
  std::vector<unsigned char> hb(bsz * (size_t)n);
  std::vector<DevTime *> ht((size_t)n);
  for (int i = 0; i < n; ++i) {
    if (fp32) memcpy(hb.data() + bsz * i, &domains[i]->bf[0], bsz);
    else memcpy(hb.data() + bsz * i, &domains[i]->bd[0], bsz);
    ht[(size_t)i] = domains[i]->time;
  }
  unsigned char *dblk = nullptr;
  if (bt->mem.get(&dblk, hb.size(), false) != cudaSuccess || bt->mem.get(&bt->times, (size_t)n, false) != cudaSuccess)
    return bad(fail(WQL3D_ENOMEM, "batch descriptors"));
  bt->blks = dblk;
  if (cudaMemcpyAsync(bt->blks, hb.data(), hb.size(), cudaMemcpyHostToDevice, bt->stream) != cudaSuccess ||
      cudaMemcpyAsync(bt->times, ht.data(), sizeof(DevTime *) * n, cudaMemcpyHostToDevice, bt->stream) != cudaSuccess)
    return bad(fail(WQL3D_ECUDA, "batch descriptor upload"));
  // classes: response x separable shell
  for (int i = 0; i < n; ++i) {
    const int sep = fp32 ? domains[i]->bf[0].sep : domains[i]->bd[0].sep;
    auto &c = bt->cls[domains[i]->response * 2 + (sep ? 1 : 0)];
    c.resp = domains[i]->response;
    c.sep = sep ? 1 : 0;
    c.shots.push_back(i);
  }
  for (auto &c : bt->cls) {
    if (c.shots.empty()) continue;
    const size_t m = c.shots.size();
    std::vector<int> shell(m + 1, 0);
    for (size_t i = 0; i < m; ++i) {
      const wql3d_domain *d = domains[c.shots[i]];
      const long long sc = fp32 ? shell_count(d->bf[0]) : shell_count(d->bd[0]);
      shell[i + 1] = shell[i] + (int)((sc + 127) / 128);
    }
    c.shell_ctas = shell.back();
    if (bt->mem.get(&c.d_shots, m, false) != cudaSuccess || bt->mem.get(&c.d_tile, m + 1, false) != cudaSuccess ||
        bt->mem.get(&c.d_shell, m + 1, false) != cudaSuccess)
      return bad(fail(WQL3D_ENOMEM, "batch work lists"));
    if (cudaMemcpyAsync(c.d_shots, c.shots.data(), sizeof(int) * m, cudaMemcpyHostToDevice, bt->stream) !=
            cudaSuccess ||
        cudaMemcpyAsync(c.d_shell, shell.data(), sizeof(int) * (m + 1), cudaMemcpyHostToDevice, bt->stream) !=
            cudaSuccess)
      return bad(fail(WQL3D_ECUDA, "batch work-list upload"));
  }
  if (const int rc = batch_tiles(bt)) return bad(rc);
  *out = bt;
  return WQL3D_OK;
}

int wql3d_batch_run(wql3d_batch *bt, double dt, int32_t nsteps, int32_t w_stride) {
  if (!bt) return fail(WQL3D_EINVAL, "null batch");
  if (nsteps <= 0) return WQL3D_OK;
  // order after the shots' own queued work, and theirs after the batch
  for (wql3d_domain *d : bt->doms) {
    CK(cudaEventRecord(bt->ev, d->stream));
    CK(cudaStreamWaitEvent(bt->stream, bt->ev, 0));
  }
  const int rc = bt->fp32 ? batch_run<float>(bt, dt, nsteps, w_stride) : batch_run<double>(bt, dt, nsteps, w_stride);
  if (rc) return rc;
  CK(cudaEventRecord(bt->ev, bt->stream));
  for (wql3d_domain *d : bt->doms) {
    CK(cudaStreamWaitEvent(d->stream, bt->ev, 0));
    d->cur = bt->cur;
  }
  return WQL3D_OK;
}

int wql3d_batch_tuning(wql3d_batch *bt, int32_t *zchunk, int32_t *ntried, int32_t *zs, float *ms) {
  if (!bt) return fail(WQL3D_EINVAL, "null batch");
  if (zchunk) *zchunk = bt->zchunk;
  if (ntried) *ntried = (int32_t)bt->tune_log.size();
  for (size_t i = 0; i < bt->tune_log.size(); ++i) {
    if (zs) zs[i] = bt->tune_log[i].first;
    if (ms) ms[i] = bt->tune_log[i].second;
  }
  return WQL3D_OK;
}

int wql3d_batch_launches(wql3d_batch *bt, int64_t *launches) {
  if (!bt || !launches) return fail(WQL3D_EINVAL, "null argument");
  *launches = bt->launches;
  return WQL3D_OK;
}

int wql3d_batch_synchronize(wql3d_batch *bt) {
  if (!bt) return fail(WQL3D_EINVAL, "null batch");
  CK(cudaStreamSynchronize(bt->stream));
  CK(cudaGetLastError());
  return WQL3D_OK;
}

int wql3d_batch_destroy(wql3d_batch *bt) {
  if (!bt) return WQL3D_OK;
  cudaStreamSynchronize(bt->stream);
  cudaStreamSynchronize(bt->side);
  if (bt->graph) cudaGraphExecDestroy(bt->graph);
  bt->mem.release();
  cudaEventDestroy(bt->fork);
  cudaEventDestroy(bt->join);
  cudaStreamDestroy(bt->side);
  cudaEventDestroy(bt->ev);
  cudaStreamDestroy(bt->stream);
  delete bt;
  return WQL3D_OK;
}

int wql3d_synchronize(wql3d_domain *d) {
  if (!d) return fail(WQL3D_EINVAL, "null domain");
  CK(cudaStreamSynchronize(d->stream));
  CK(cudaGetLastError());
  return WQL3D_OK;
}

int wql3d_get_stream(wql3d_domain *d, void **stream) {
  if (!d || !stream) return fail(WQL3D_EINVAL, "null argument");
  *stream = (void *)d->stream;
  return WQL3D_OK;
}

int wql3d_device_bytes(wql3d_domain *d, int64_t *bytes) {
  if (!d || !bytes) return fail(WQL3D_EINVAL, "null argument");
  *bytes = d->mem.bytes;
  return WQL3D_OK;
}

int wql3d_kernel_launches(wql3d_domain *d, int64_t *launches) {
  if (!d || !launches) return fail(WQL3D_EINVAL, "null argument");
  *launches = d->launches;
  return WQL3D_OK;
}

}  // extern "C"
