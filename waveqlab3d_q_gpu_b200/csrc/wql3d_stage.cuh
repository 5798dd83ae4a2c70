// Host-side launchers of the per-block stage kernels, one family per
// translation unit (stage_cart.cu, stage_curv.cu, stage_generic.cu), each
// compiled once per precision (WQL3D_REAL = double / float) so that the
// heavy kernel templates build in parallel.  wql3d_api.cu calls them through
// the declarations below.
//
// __constant__ tables are per translation unit (no relocatable device code):
// every family TU exports an uploader that copies the SBP rows and the RK
// coefficients into its own copy.
#pragma once

#include <cstdint>
#include <cstdlib>
#include <cstring>

#include "wql3d_device.cuh"

namespace wql3d {

struct ConstTables {
  int sbp_cnt[6];
  int sbp_idx[6][8];
  double sbp_c[2][6][8];
  double rkA[5], rkB[5], rkC[6];
};

// per-stage launch context of one block
struct StageCtx {
  cudaStream_t stream;
  int response;       // RESP_*
  int64_t *launches;  // kernel-launch counter of the owning domain
  // optional second stream and fork / join events: the Cartesian shell runs
  // there, concurrently with the interior (disjoint points, read-only F)
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};

// tuning switches read once per translation unit from the environment
struct Tuning {
  int zchunk = 12;    // z planes per Cartesian interior tile
  int generic = 0;    // 1: every point through the generic per-point kernel
  int lean = 1;       // curvilinear update: k_curv_point (0: generic point update k_curv_update)
  int curv_fused = 1; // curvilinear stage in one pass, k_curv_fused (0: derivative / memory-variable / point passes)
  int fused_minb = 0; // k_curv_fused resident 128-thread blocks per SM: 3 (default), 2 or 4 in FP64; 4 (default), 5 or 6 in FP32
  int mvpf = -1;      // k_curv_fused: L2 prefetch of the memory variables on entry (-1: FP32 only)
  int overlap = 1;    // Cartesian stage: shell on the side stream, concurrent with the interior
  int tma = 0;        // Cartesian interior: 1 = planes filled by TMA box loads (default: cp.async, measured faster);
                      // 2 = TMA waits with no copies issued (test of the bounded waits and the stall status)
};

inline Tuning tuning() {
  static Tuning t = [] {
    Tuning r;
    if (const char *e = getenv("WQL3D_ZCHUNK")) r.zchunk = atoi(e) > 0 ? atoi(e) : 1;
    if (const char *e = getenv("WQL3D_FUSED_MINB")) r.fused_minb = atoi(e);
    if (const char *e = getenv("WQL3D_MV_PREFETCH")) r.mvpf = atoi(e);
    if (const char *e = getenv("WQL3D_SHELL_OVERLAP")) r.overlap = atoi(e);
    if (const char *e = getenv("WQL3D_TMA")) r.tma = atoi(e);
    if (const char *e = getenv("WQL3D_KERNEL")) {
      r.generic = strcmp(e, "generic") == 0;
      if (strcmp(e, "curv_generic_update") == 0) r.lean = 0;
      if (strcmp(e, "curv_split") == 0) r.curv_fused = 0;
    }
    return r;
  }();
  return t;
}

// copy the tables into this translation unit's __constant__ memory
inline int upload_tables_here(const ConstTables &t) {
  cudaError_t e = cudaMemcpyToSymbol(c_sbp_cnt, t.sbp_cnt, sizeof(t.sbp_cnt));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_sbp_idx, t.sbp_idx, sizeof(t.sbp_idx));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_sbp_c, t.sbp_c, sizeof(t.sbp_c));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_rkA, t.rkA, sizeof(t.rkA));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_rkB, t.rkB, sizeof(t.rkB));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_rkC, t.rkC, sizeof(t.rkC));
  return (int)e;
}

// Cartesian fused stage (flags == F_ALL): strict interior + near-boundary shell
template <typename T>
void launch_cart_stage(Blk<T> &b, const StageCtx &c, const StageArgs &a);
// curvilinear split stage: derivative pass, memory variables, face SATs, point update
template <typename T>
void launch_curv_stage(Blk<T> &b, const StageCtx &c, const StageArgs &a);
// true when the block's full curvilinear stages run k_curv_fused (which can
// record the adjoint's derivative terms, StageArgs::rec)
template <typename T>
bool curv_stage_fused(const Blk<T> &b);
// generic per-point kernel (any flags, MMS, both meshes)
template <typename T>
void launch_generic_stage(Blk<T> &b, int mesh, const StageCtx &c, const StageArgs &a);

int upload_tables_cart_f64(const ConstTables &t);
int upload_tables_cart_f32(const ConstTables &t);
int upload_tables_curv_f64(const ConstTables &t);
int upload_tables_curv_f32(const ConstTables &t);
int upload_tables_generic_f64(const ConstTables &t);
int upload_tables_generic_f32(const ConstTables &t);

}  // namespace wql3d

// one family TU: WQL3D_REAL (double or float) and WQL3D_TAG (f64 or f32) come
// from the compile line
#define WQL3D_CAT2(a, b) a##b
#define WQL3D_CAT(a, b) WQL3D_CAT2(a, b)
