// Block-interface coupling on the q-direction interface between two blocks.
#pragma once

#include <vector>

#include "wql3d.h"
#include "wql3d_device.cuh"

namespace wql3d {

struct IfaceDev {
  int ny = 0, nz = 0;
  void *sat_m = nullptr;   // SAT vector added at block 1's q-max face (F_x)
  void *sat_p = nullptr;   // SAT vector added at block 2's q-min face (G_x)
};

template <typename T>
int setup_iface(IfaceDev &I, const wql3d_domain_desc &desc, Blk<T> &b0, Blk<T> &b1, std::vector<void *> &ptrs,
                int64_t &bytes, cudaStream_t s) {
  (void)I; (void)desc; (void)b0; (void)b1; (void)ptrs; (void)bytes; (void)s;
  return WQL3D_EINVAL;
}

template <typename T>
void launch_iface(IfaceDev &I, const Blk<T> &b0, const Blk<T> &b1, const StageArgs &a, cudaStream_t s) {
  (void)I; (void)b0; (void)b1; (void)a; (void)s;
}

template <typename T>
void launch_iface_update(IfaceDev &I, const StageArgs &a, cudaStream_t s) { (void)I; (void)a; (void)s; }

inline void iface_scale(IfaceDev &I, double A, cudaStream_t s) { (void)I; (void)A; (void)s; }

inline int iface_download(IfaceDev &I, double *out, cudaStream_t s) { (void)I; (void)out; (void)s; return WQL3D_EINVAL; }

}  // namespace wql3d
