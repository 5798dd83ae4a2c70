// Curvilinear block mesh on the device: 3-D transfinite interpolation of the
// six boundary surfaces, Gen3_Curve_Mesh of src/grid.f90:2292-2418 (the
// O(n^3) part of Curve_Grid_3D3, src/grid.f90:473-1909; the 2-D surfaces are
// built by the caller).
#include <cuda_runtime.h>

#include <string>

#include "wql3d.h"

namespace wql3d {
void set_last_error(const std::string &msg);  // wql3d_api.cu: text returned by wql3d_last_error()
}

namespace {

// faces: left, right (3 x ns x nr), top, bottom (3 x ns x nq), front, back
// (3 x nr x nq), first index slowest; out: 3 x ns x nr x nq (q fastest)
__global__ void k_tfi(const double *__restrict__ faces, int nq, int nr, int ns, double *__restrict__ out) {
  const long long npt = (long long)nq * nr * ns;
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= npt) return;
  const int i = (int)(p % nq), j = (int)((p / nq) % nr), k = (int)(p / ((long long)nq * nr));
  const long long nLR = 3LL * ns * nr, nTB = 3LL * ns * nq;
  const double *Lf = faces, *Rf = Lf + nLR, *Tf = Rf + nLR, *Bf = Tf + nTB, *Ff = Bf + nTB, *Kf = Ff + 3LL * nr * nq;
  const double hq = 1.0 / (double)(nq - 1), hr = 1.0 / (double)(nr - 1), hs = 1.0 / (double)(ns - 1);
  const double q = (double)i * hq, r = (double)j * hr, s = (double)k * hs;
  for (int c = 0; c < 3; ++c) {
    // face accessors in the reference's (first, second) index order
    auto L = [&](int jj, int kk) { return Lf[((long long)c * ns + kk) * nr + jj]; };
    auto R = [&](int jj, int kk) { return Rf[((long long)c * ns + kk) * nr + jj]; };
    auto T = [&](int ii, int kk) { return Tf[((long long)c * ns + kk) * nq + ii]; };
    auto B = [&](int ii, int kk) { return Bf[((long long)c * ns + kk) * nq + ii]; };
    auto F = [&](int ii, int jj) { return Ff[((long long)c * nr + jj) * nq + ii]; };
    auto K = [&](int ii, int jj) { return Kf[((long long)c * nr + jj) * nq + ii]; };
    const double U = (1.0 - q) * L(j, k) + q * R(j, k);
    const double V = (1.0 - r) * T(i, k) + r * B(i, k);
    const double W = (1.0 - s) * F(i, j) + s * K(i, j);
    const double UW = (1.0 - q) * ((1.0 - r) * L(0, k) + r * L(nr - 1, k)) + q * ((1.0 - r) * R(0, k) + r * R(nr - 1, k));
    const double UV = (1.0 - r) * ((1.0 - s) * T(i, 0) + s * T(i, ns - 1)) + r * ((1.0 - s) * B(i, 0) + s * B(i, ns - 1));
    const double VW = (1.0 - s) * ((1.0 - q) * F(0, j) + q * F(nq - 1, j)) + s * ((1.0 - q) * K(0, j) + q * K(nq - 1, j));
    const double UVW1 = (1.0 - q) * ((1.0 - r) * ((1.0 - s) * T(0, 0) + s * T(0, ns - 1)) +
                                     r * ((1.0 - s) * B(0, 0) + s * B(0, ns - 1)));
    const double UVW2 = q * ((1.0 - r) * ((1.0 - s) * T(nq - 1, 0) + s * T(nq - 1, ns - 1)) +
                             r * ((1.0 - s) * B(nq - 1, 0) + s * B(nq - 1, ns - 1)));
    out[(long long)c * npt + p] = U + V + W - UV - UW - VW + UVW1 + UVW2;
  }
}

}  // namespace

extern "C" int wql3d_tfi_grid(const double *faces, int32_t nq, int32_t nr, int32_t ns, double *coords) {
  if (!faces || !coords || nq < 2 || nr < 2 || ns < 2) {
    wql3d::set_last_error("wql3d_tfi_grid: null array or fewer than 2 points on an axis");
    return WQL3D_EINVAL;
  }
  const size_t nf = 3 * (2 * (size_t)ns * nr + 2 * (size_t)ns * nq + 2 * (size_t)nr * nq);
  const size_t no = 3 * (size_t)nq * nr * ns;
  double *df = nullptr, *dout = nullptr;
  cudaError_t e = cudaMalloc(&df, nf * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&dout, no * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpy(df, faces, nf * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    const long long npt = (long long)nq * nr * ns;
    k_tfi<<<(unsigned)((npt + 255) / 256), 256>>>(df, nq, nr, ns, dout);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(coords, dout, no * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(df);
  cudaFree(dout);
  if (e != cudaSuccess) {
    wql3d::set_last_error(std::string("wql3d_tfi_grid: ") + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? WQL3D_ENOMEM : WQL3D_ECUDA;
  }
  return WQL3D_OK;
}
