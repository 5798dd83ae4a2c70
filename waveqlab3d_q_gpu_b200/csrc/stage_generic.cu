// Generic per-point stage launcher (any stage flags, manufactured solutions,
// both meshes), compiled once per precision.
#include "wql3d_stage.cuh"

namespace wql3d {

template <typename T>
void launch_generic_stage(Blk<T> &b, int mesh, const StageCtx &c, const StageArgs &a) {
  dim3 th(32, 4, 2), gr((b.nx + 31) / 32, (b.ny + 3) / 4, (b.nz + 1) / 2);
  switch (c.response * 2 + mesh) {
    case 0: k_stage<T, MESH_CART, RESP_EL><<<gr, th, 0, c.stream>>>(b, a); break;
    case 1: k_stage<T, MESH_CURV, RESP_EL><<<gr, th, 0, c.stream>>>(b, a); break;
    case 2: k_stage<T, MESH_CART, RESP_Q4><<<gr, th, 0, c.stream>>>(b, a); break;
    case 3: k_stage<T, MESH_CURV, RESP_Q4><<<gr, th, 0, c.stream>>>(b, a); break;
    case 4: k_stage<T, MESH_CART, RESP_Q8><<<gr, th, 0, c.stream>>>(b, a); break;
    case 5: k_stage<T, MESH_CURV, RESP_Q8><<<gr, th, 0, c.stream>>>(b, a); break;
    case 6: k_stage<T, MESH_CART, RESP_FQ8><<<gr, th, 0, c.stream>>>(b, a); break;
    default: k_stage<T, MESH_CURV, RESP_FQ8><<<gr, th, 0, c.stream>>>(b, a); break;
  }
  ++*c.launches;
}

template void launch_generic_stage<WQL3D_REAL>(Blk<WQL3D_REAL> &, int, const StageCtx &, const StageArgs &);
int WQL3D_CAT(upload_tables_generic_, WQL3D_TAG)(const ConstTables &t) { return upload_tables_here(t); }

}  // namespace wql3d
