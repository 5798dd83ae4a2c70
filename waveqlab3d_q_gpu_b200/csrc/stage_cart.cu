// Cartesian fused stage launcher (strict interior + near-boundary shell),
// compiled once per precision.
#include "wql3d_stage.cuh"

namespace wql3d {

template <typename T, int RESP>
static void launch_interior(Blk<T> &b, const StageCtx &c, const StageArgs &a) {
  const int zchunk = tuning().zchunk;
  int nxi = b.hi[0] - b.lo[0] + 1, nyi = b.hi[1] - b.lo[1] + 1, nzi = b.hi[2] - b.lo[2] + 1;
  if (nxi <= 0 || nyi <= 0 || nzi <= 0) return;
  dim3 gr((nxi + 31) / 32, (nyi + 3) / 4, (nzi + zchunk - 1) / zchunk);
  size_t sm = SplitSmem<T, 4>::bytes;
  cudaFuncSetAttribute(k_interior_split<T, RESP, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_interior_split<T, RESP, 4><<<gr, 256, sm, c.stream>>>(b, a, zchunk);
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
