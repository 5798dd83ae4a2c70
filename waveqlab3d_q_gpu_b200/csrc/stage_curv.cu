// Curvilinear stage launcher: derivative pass, memory-variable pass, face-SAT
// pre-pass and point update (or the generic point update where a block's two
// PML slabs on one axis overlap), compiled once per precision.
#include "wql3d_stage.cuh"

namespace wql3d {

// fused stage: face-SAT pre-pass, then one pass over every point with the
// derivative terms and memory-variable sums in registers; MB resident blocks
// of 128 threads per SM
template <typename T, int MB>
static void launch_fused_mb(Blk<T> &b, const StageCtx &c, const StageArgs &a, unsigned gr) {
  switch (c.response) {
    case RESP_EL: k_curv_fused<T, RESP_EL, MB><<<gr, 128, 0, c.stream>>>(b, a); break;
    case RESP_Q4: k_curv_fused<T, RESP_Q4, MB><<<gr, 128, 0, c.stream>>>(b, a); break;
    case RESP_Q8: k_curv_fused<T, RESP_Q8, MB><<<gr, 128, 0, c.stream>>>(b, a); break;
    default: k_curv_fused<T, RESP_FQ8, MB><<<gr, 128, 0, c.stream>>>(b, a); break;
  }
}

template <typename T>
static void launch_curv_fused(Blk<T> &b, const StageCtx &c, const StageArgs &a) {
  const long long npts = (long long)b.nx * b.ny * b.nz;
  if ((a.flags & F_SAT) && b.foff[6] > 0) {
    k_curv_face_sat<T><<<(b.foff[6] + 127) / 128, 128, 0, c.stream>>>(b, a.cur);
    ++*c.launches;
  }
  const unsigned gr = (unsigned)((npts + 127) / 128);
  const int mb = tuning().fused_minb;
  StageArgs la = a;
  // L2 prefetch of the memory variables: on by default in FP32 only (measured
  // 2.7 % faster there, 4.5 % slower in FP64)
  la.pf = tuning().mvpf >= 0 ? tuning().mvpf : (sizeof(T) == 4 ? 1 : 0);
  if (sizeof(T) == 8) {
    if (mb == 2) launch_fused_mb<T, 2>(b, c, la, gr);
    else if (mb == 4) launch_fused_mb<T, 4>(b, c, la, gr);
    else launch_fused_mb<T, 3>(b, c, la, gr);
  } else {
    if (mb == 6) launch_fused_mb<T, 6>(b, c, la, gr);
    else if (mb == 5) launch_fused_mb<T, 5>(b, c, la, gr);
    else launch_fused_mb<T, 4>(b, c, la, gr);
  }
  ++*c.launches;
}

// the lean kernels keep one PML slab per axis: blocks whose two slabs on an
// axis overlap (2 npml > n) take the generic update
template <typename T>
static bool pml_overlap(const Blk<T> &b) {
  const int nax[3] = {b.nx, b.ny, b.nz};
  for (int ax = 0; ax < 3; ++ax)
    if (b.pml_on[2 * ax] && b.pml_on[2 * ax + 1] && 2 * b.npml > nax[ax]) return true;
  return false;
}

template <typename T>
bool curv_stage_fused(const Blk<T> &b) {
  return tuning().curv_fused && tuning().lean && !pml_overlap(b);
}

template <typename T>
void launch_curv_stage(Blk<T> &b, const StageCtx &c, const StageArgs &a) {
  const long long npts = (long long)b.nx * b.ny * b.nz;
  const bool overlap = pml_overlap(b);
  if (curv_stage_fused(b)) {
    launch_curv_fused<T>(b, c, a);
    return;
  }
  if (a.flags & F_RHS) {
    const unsigned fgr = (unsigned)((npts + 255) / 256);
    k_curv_grad<T, 2, 1><<<fgr, 256, 0, c.stream>>>(b, a.cur);
    ++*c.launches;
  }
  if (!tuning().lean || overlap) {
    dim3 th(32, 4, 2), gr((b.nx + 31) / 32, (b.ny + 3) / 4, (b.nz + 1) / 2);
    switch (c.response) {
      case RESP_EL: k_curv_update<T, RESP_EL><<<gr, th, 0, c.stream>>>(b, a); break;
      case RESP_Q4: k_curv_update<T, RESP_Q4><<<gr, th, 0, c.stream>>>(b, a); break;
      case RESP_Q8: k_curv_update<T, RESP_Q8><<<gr, th, 0, c.stream>>>(b, a); break;
      default: k_curv_update<T, RESP_FQ8><<<gr, th, 0, c.stream>>>(b, a); break;
    }
    ++*c.launches;
    return;
  }
  if (c.response != RESP_EL && (a.flags & (F_RHS | F_SCALE | F_UPDATE))) {
    // memory variables first: k_curv_point subtracts their sums; 3 (FP64) or
    // 8 (FP32) resident blocks of 128 threads
    constexpr int AMINB = sizeof(T) == 4 ? 8 : 3;
    const unsigned agr = (unsigned)((npts + 127) / 128);
    switch (c.response) {
      case RESP_Q4: k_curv_anelastic<T, RESP_Q4, AMINB><<<agr, 128, 0, c.stream>>>(b, a); break;
      case RESP_Q8: k_curv_anelastic<T, RESP_Q8, AMINB><<<agr, 128, 0, c.stream>>>(b, a); break;
      default: k_curv_anelastic<T, RESP_FQ8, AMINB><<<agr, 128, 0, c.stream>>>(b, a); break;
    }
    ++*c.launches;
  }
  if ((a.flags & F_SAT) && b.foff[6] > 0) {
    k_curv_face_sat<T><<<(b.foff[6] + 127) / 128, 128, 0, c.stream>>>(b, a.cur);
    ++*c.launches;
  }
  // point update: 256 threads, 2 (FP64) or 4 (FP32) resident blocks
  constexpr int PMINB = sizeof(T) == 4 ? 4 : 2;
  const unsigned gr = (unsigned)((npts + 255) / 256);
  switch (c.response) {
    case RESP_EL: k_curv_point<T, RESP_EL, 256, PMINB><<<gr, 256, 0, c.stream>>>(b, a); break;
    case RESP_Q4: k_curv_point<T, RESP_Q4, 256, PMINB><<<gr, 256, 0, c.stream>>>(b, a); break;
    case RESP_Q8: k_curv_point<T, RESP_Q8, 256, PMINB><<<gr, 256, 0, c.stream>>>(b, a); break;
    default: k_curv_point<T, RESP_FQ8, 256, PMINB><<<gr, 256, 0, c.stream>>>(b, a); break;
  }
  ++*c.launches;
}

template void launch_curv_stage<WQL3D_REAL>(Blk<WQL3D_REAL> &, const StageCtx &, const StageArgs &);
template bool curv_stage_fused<WQL3D_REAL>(const Blk<WQL3D_REAL> &);
int WQL3D_CAT(upload_tables_curv_, WQL3D_TAG)(const ConstTables &t) { return upload_tables_here(t); }

}  // namespace wql3d
