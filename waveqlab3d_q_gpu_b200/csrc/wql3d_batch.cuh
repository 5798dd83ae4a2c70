// Batched independent shots (stage_batch.cu): work-list descriptors and the
// host launchers.  No counterpart in the reference, which runs one problem per
// process.
#pragma once

#include "wql3d_stage.cuh"

namespace wql3d {

// one class of shots launched together: same response and near-boundary
// variant (separable or full-metric shell)
template <typename T>
struct BatchClass {
  int resp, sep;
  int nshots;              // shots of this class
  const int *shots;        // their indices in the batch
  const int *tile_prefix;  // interior CTAs: nshots + 1 offsets
  const int *shell_prefix; // shell CTAs (128 points each): nshots + 1 offsets
  int tiles, shell_ctas;   // totals
  const Blk<T> *blks;      // every shot's block descriptor (device)
  DevTime *const *times;   // every shot's step time / sample counter (device)
};

// side != nullptr: the shells run on the side stream (fork / join events),
// concurrently with the interior tiles
template <typename T>
void launch_batch_stage(const BatchClass<T> *classes, int ncls, const StageArgs &a, int zchunk, cudaStream_t s,
                        cudaStream_t side, cudaEvent_t fork, cudaEvent_t join, int64_t *launches);
template <typename T>
void launch_batch_sample(const Blk<T> *blks, DevTime *const *times, int nshots, int cur, int w_stride,
                         cudaStream_t s, int64_t *launches);
template <typename T>
void launch_batch_advance(DevTime *const *times, int nshots, double dt, cudaStream_t s, int64_t *launches);

int upload_tables_batch_f64(const ConstTables &t);
int upload_tables_batch_f32(const ConstTables &t);

}  // namespace wql3d
