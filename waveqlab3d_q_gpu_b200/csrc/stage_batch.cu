// Batched independent shots: one launch per kernel kind covers every shot of
// a class (same response, same near-boundary variant), compiled once per
// precision.  A shot is a one-block Cartesian domain; the batch holds the
// shots' block descriptors in device memory and each CTA stages its shot's
// descriptor in shared memory before running the same tile / point bodies as
// the per-domain kernels (interior_split_tile, point_update, sample_block).
//
// Work lists: every CTA belongs to one shot.  The interior launch covers the
// shots' 32 x 4 x zchunk tiles, the shell launch their near-boundary points
// in chunks of 128 (each shot's chunk count rounded up, so no CTA straddles
// two shots); a prefix array over the class's shots maps a CTA to its shot.
#include "wql3d_batch.cuh"

namespace wql3d {

namespace {

// shot of CTA c in a prefix array of n + 1 CTA offsets (binary search)
__device__ __forceinline__ int owner(const int *prefix, int n, int c) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(prefix + mid) <= c) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// copy one shot's block descriptor into shared memory (all threads take part)
template <typename T>
__device__ __forceinline__ void stage_blk(const Blk<T> *src, Blk<T> *dst) {
  const unsigned long long *s = reinterpret_cast<const unsigned long long *>(src);
  unsigned long long *d = reinterpret_cast<unsigned long long *>(dst);
  constexpr int nw = (int)(sizeof(Blk<T>) / sizeof(unsigned long long));
  for (int i = threadIdx.x; i < nw; i += blockDim.x) d[i] = s[i];
}

template <typename T, int RESP>
__global__ void __launch_bounds__(256, 2) k_batch_interior(BatchClass<T> C, StageArgs a, int zchunk) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ __align__(16) Blk<T> sb;
  __shared__ int s_shot, s_local;
  if (threadIdx.x == 0) {
    const int k = owner(C.tile_prefix, C.nshots, blockIdx.x);
    s_shot = C.shots[k];
    s_local = blockIdx.x - C.tile_prefix[k];
  }
  __syncthreads();
  stage_blk<T>(C.blks + s_shot, &sb);
  __syncthreads();
  const int ntx = (sb.hi[0] - sb.lo[0] + 32) / 32, nty = (sb.hi[1] - sb.lo[1] + 4) / 4;
  const int bx = s_local % ntx, by = (s_local / ntx) % nty, bz = s_local / (ntx * nty);
  StageArgs la = a;
  la.time = C.times[s_shot];
  interior_split_tile<T, RESP, 4>(sb, la, zchunk, bx, by, bz, smraw);
}

template <typename T, int RESP, bool SEP>
__global__ void __launch_bounds__(128, 3) k_batch_shell(BatchClass<T> C, StageArgs a) {
  __shared__ __align__(16) Blk<T> sb;
  __shared__ int s_shot, s_local;
  if (threadIdx.x == 0) {
    const int k = owner(C.shell_prefix, C.nshots, blockIdx.x);
    s_shot = C.shots[k];
    s_local = blockIdx.x - C.shell_prefix[k];
  }
  __syncthreads();
  stage_blk<T>(C.blks + s_shot, &sb);
  __syncthreads();
  const long long idx = (long long)s_local * 128 + threadIdx.x;
  if (idx >= shell_count(sb)) return;
  int x, y, z;
  shell_decode(sb, (int)idx, x, y, z);
  StageArgs la = a;
  la.time = C.times[s_shot];
  point_update<T, MESH_CART, RESP, SEP, false, true>(sb, la, x, y, z);
}

// stage-1 station samples of every shot: one CTA per shot
template <typename T>
__global__ void __launch_bounds__(256) k_batch_sample(const Blk<T> *blks, DevTime *const *times, int cur,
                                                      int w_stride) {
  __shared__ __align__(16) Blk<T> sb;
  stage_blk<T>(blks + blockIdx.x, &sb);
  __syncthreads();
  if (sb.nrec > 0) sample_block<T>(sb, cur, times[blockIdx.x], w_stride, 1);
}

// every shot's time advance after its fifth stage (templated on the precision
// so the two compilations of this file define distinct kernels)
template <typename T>
__global__ void k_batch_advance(DevTime *const *times, int n, double dt) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  DevTime *tm = times[s];
  tm->t = tm->t + c_rkC[5] * dt;
  tm->n = tm->n + 1;
}

// interior tiles (part 0) or near-boundary shell (part 1) of one class
template <typename T, int RESP>
void launch_class(const BatchClass<T> &C, const StageArgs &a, int zchunk, cudaStream_t s, int part,
                  int64_t *launches) {
  if (part == 0 && C.tiles > 0) {
    const size_t sm = SplitSmem<T, 4>::bytes;
    cudaFuncSetAttribute(k_batch_interior<T, RESP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_batch_interior<T, RESP><<<C.tiles, 256, sm, s>>>(C, a, zchunk);
    ++*launches;
  }
  if (part == 1 && C.shell_ctas > 0) {
    if (C.sep) k_batch_shell<T, RESP, true><<<C.shell_ctas, 128, 0, s>>>(C, a);
    else k_batch_shell<T, RESP, false><<<C.shell_ctas, 128, 0, s>>>(C, a);
    ++*launches;
  }
}

template <typename T>
void launch_part(const BatchClass<T> *classes, int ncls, const StageArgs &a, int zchunk, cudaStream_t s, int part,
                 int64_t *launches) {
  for (int c = 0; c < ncls; ++c) {
    const BatchClass<T> &C = classes[c];
    if (C.nshots == 0) continue;
    switch (C.resp) {
      case RESP_EL: launch_class<T, RESP_EL>(C, a, zchunk, s, part, launches); break;
      case RESP_Q4: launch_class<T, RESP_Q4>(C, a, zchunk, s, part, launches); break;
      case RESP_Q8: launch_class<T, RESP_Q8>(C, a, zchunk, s, part, launches); break;
      default: launch_class<T, RESP_FQ8>(C, a, zchunk, s, part, launches); break;
    }
  }
}

}  // namespace

template <typename T>
void launch_batch_stage(const BatchClass<T> *classes, int ncls, const StageArgs &a, int zchunk, cudaStream_t s,
                        cudaStream_t side, cudaEvent_t fork, cudaEvent_t join, int64_t *launches) {
  if (side) {
    // every class's shell on the side stream, next to the interior tiles
    // (disjoint points of independent shots)
    cudaEventRecord(fork, s);
    cudaStreamWaitEvent(side, fork, 0);
    launch_part<T>(classes, ncls, a, zchunk, side, 1, launches);
    cudaEventRecord(join, side);
    launch_part<T>(classes, ncls, a, zchunk, s, 0, launches);
    cudaStreamWaitEvent(s, join, 0);
    return;
  }
  launch_part<T>(classes, ncls, a, zchunk, s, 0, launches);
  launch_part<T>(classes, ncls, a, zchunk, s, 1, launches);
}

template <typename T>
void launch_batch_sample(const Blk<T> *blks, DevTime *const *times, int nshots, int cur, int w_stride,
                         cudaStream_t s, int64_t *launches) {
  k_batch_sample<T><<<nshots, 256, 0, s>>>(blks, times, cur, w_stride);
  ++*launches;
}

template <typename T>
void launch_batch_advance(DevTime *const *times, int nshots, double dt, cudaStream_t s, int64_t *launches) {
  k_batch_advance<T><<<(nshots + 127) / 128, 128, 0, s>>>(times, nshots, dt);
  ++*launches;
}

template void launch_batch_stage<WQL3D_REAL>(const BatchClass<WQL3D_REAL> *, int, const StageArgs &, int,
                                             cudaStream_t, cudaStream_t, cudaEvent_t, cudaEvent_t, int64_t *);
template void launch_batch_sample<WQL3D_REAL>(const Blk<WQL3D_REAL> *, DevTime *const *, int, int, int,
                                              cudaStream_t, int64_t *);
template void launch_batch_advance<WQL3D_REAL>(DevTime *const *, int, double, cudaStream_t, int64_t *);
int WQL3D_CAT(upload_tables_batch_, WQL3D_TAG)(const ConstTables &t) { return upload_tables_here(t); }

}  // namespace wql3d
