// Cartesian fused stage launcher (strict interior + near-boundary shell),
// compiled once per precision.
#include <cudaTypedefs.h>

#include "wql3d_stage.cuh"

namespace wql3d {

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library)
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// 4-D tensor map (x, y, z, component) of the field buffer F with the interior
// tile's W x H x 1 x 1 box (zero fill outside the padded array); false when
// the layout breaks a TMA rule (the tile then fills its planes with cp.async)
template <typename T>
static bool plane_tensor_map(const Blk<T> &b, const T *F, CUtensorMap *m) {
  using SM = SplitSmem<T, 4>;
  const auto enc = tensor_map_encoder();
  if (!enc || !F) return false;
  const cuuint64_t esz = sizeof(T);
  if ((reinterpret_cast<uintptr_t>(F) & 15) || (b.sy * esz) % 16 || (b.sz * esz) % 16 || (b.vol * esz) % 16 ||
      (SM::W * esz) % 16 || SM::W > 256 || SM::H > 256)
    return false;
  cuuint64_t dims[4] = {(cuuint64_t)b.sy, (cuuint64_t)(b.sz / b.sy), (cuuint64_t)(b.vol / b.sz), 9};
  cuuint64_t strides[3] = {(cuuint64_t)b.sy * esz, (cuuint64_t)b.sz * esz, (cuuint64_t)b.vol * esz};
  cuuint32_t box[4] = {(cuuint32_t)SM::W, (cuuint32_t)SM::H, 1, 1};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  const CUresult r = enc(m, sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                         const_cast<T *>(F), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <typename T, int RESP>
static void launch_interior(Blk<T> &b, const StageCtx &c, const StageArgs &a) {
  const int zchunk = tuning().zchunk;
  int nxi = b.hi[0] - b.lo[0] + 1, nyi = b.hi[1] - b.lo[1] + 1, nzi = b.hi[2] - b.lo[2] + 1;
  if (nxi <= 0 || nyi <= 0 || nzi <= 0) return;
  dim3 gr((nxi + 31) / 32, (nyi + 3) / 4, (nzi + zchunk - 1) / zchunk);
  CUtensorMap tm;
  memset(&tm, 0, sizeof(tm));
  if (tuning().tma && plane_tensor_map<T>(b, a.cur ? b.F1 : b.F0, &tm)) {
    const size_t sm = SplitSmem<T, 4>::bytes;
    StageArgs ta = a;
    ta.nofill = tuning().tma == 2;
    cudaFuncSetAttribute(k_interior_split<T, RESP, 4, true, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_interior_split<T, RESP, 4, true, 2><<<gr, 256, sm, c.stream>>>(b, ta, zchunk, tm);
  } else {
    const size_t sm = SplitSmem<T, 4>::bytes;
    cudaFuncSetAttribute(k_interior_split<T, RESP, 4, false, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_interior_split<T, RESP, 4, false, 2><<<gr, 256, sm, c.stream>>>(b, a, zchunk, tm);
  }
  ++*c.launches;
}

template <typename T, int RESP>
static void launch_shell(Blk<T> &b, const StageCtx &c, const StageArgs &a) {
  long long n = shell_count(b);
  if (n <= 0) return;
  unsigned g = (unsigned)((n + 127) / 128);
  if (b.sep) k_shell<T, MESH_CART, RESP, true><<<g, 128, 0, c.stream>>>(b, a, (int)n);
  else k_shell<T, MESH_CART, RESP, false><<<g, 128, 0, c.stream>>>(b, a, (int)n);
  ++*c.launches;
}

template <typename T, int RESP>
static void launch_both(Blk<T> &b, const StageCtx &c, const StageArgs &a) {
  if (c.side && tuning().overlap) {
    // the shell (latency-bound, one thread per scattered point) on the side
    // stream next to the bandwidth-bound interior tiles; both read the
    // current fields and write disjoint points
    StageCtx sc = c;
    sc.stream = c.side;
    cudaEventRecord(c.fork, c.stream);
    cudaStreamWaitEvent(c.side, c.fork, 0);
    launch_shell<T, RESP>(b, sc, a);
    cudaEventRecord(c.join, c.side);
    launch_interior<T, RESP>(b, c, a);
    cudaStreamWaitEvent(c.stream, c.join, 0);
    return;
  }
  launch_interior<T, RESP>(b, c, a);
  launch_shell<T, RESP>(b, c, a);
}

template <typename T>
void launch_cart_stage(Blk<T> &b, const StageCtx &c, const StageArgs &a) {
  switch (c.response) {
    case RESP_EL: launch_both<T, RESP_EL>(b, c, a); break;
    case RESP_Q4: launch_both<T, RESP_Q4>(b, c, a); break;
    case RESP_Q8: launch_both<T, RESP_Q8>(b, c, a); break;
    default: launch_both<T, RESP_FQ8>(b, c, a); break;
  }
}

template void launch_cart_stage<WQL3D_REAL>(Blk<WQL3D_REAL> &, const StageCtx &, const StageArgs &);
int WQL3D_CAT(upload_tables_cart_, WQL3D_TAG)(const ConstTables &t) { return upload_tables_here(t); }

}  // namespace wql3d
