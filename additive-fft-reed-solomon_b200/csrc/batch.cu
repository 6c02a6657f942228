// Batched path: many independent codewords of different shapes (n, t,
// shard length, erasure pattern, encode or recover) in one persistent
// launch driven by a per-codeword descriptor table.
//
// Work is split into tasks (codeword, 256-column tile); persistent CTAs take
// tasks from a global counter, so short and long codewords balance across
// the SMs.  Each task runs the generic tile routines (runtime twiddles), so
// one kernel serves every shape.  Recover jobs get their erasure locator
// from a pre-pass (one CTA per recover job).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "afrs_internal.h"
#include "generic_tile.cuh"

namespace afrs {
namespace {

using namespace gtile;

constexpr int kLocBytes = 768;  // erased flags, lambda values, 1/lambda' values

__global__ void __launch_bounds__(kThreads) k_batch_locator(const BatchJob* jobs, const int* rec_jobs,
                                                             const uint8_t* pos_tab, uint8_t* loc_tab) {
  __shared__ uint8_t s_er[256], s_lam[256], s_ilp[256];
  __shared__ int s_x[256], s_y[256];
  const BatchJob jb = jobs[rec_jobs[blockIdx.x]];
  erasure_locator(jb.n, jb.e, pos_tab + jb.pos_off, s_er, s_lam, s_ilp, s_x, s_y);
  uint8_t* out = loc_tab + (size_t)jb.loc * kLocBytes;
  for (int i = threadIdx.x; i < 256; i += blockDim.x) {
    out[i] = i < jb.n ? s_er[i] : 0;
    out[256 + i] = i < jb.n ? s_lam[i] : 0;
    out[512 + i] = i < jb.n ? s_ilp[i] : 0;
  }
}

__global__ void __launch_bounds__(kThreads) k_batch(const BatchJob* jobs, const uint2* tasks, int ntasks,
                                                     unsigned* counter, const uint8_t* pos_tab,
                                                     const uint8_t* loc_tab) {
  extern __shared__ uint32_t sm[];
  __shared__ uint8_t s_er[256], s_lam[256], s_ilp[256];
  __shared__ int s_task;
  for (;;) {
    if (threadIdx.x == 0) s_task = (int)atomicAdd(counter, 1u);
    __syncthreads();
    const int tk = s_task;
    if (tk >= ntasks) break;
    const uint2 task = tasks[tk];
    const BatchJob jb = jobs[task.x];
    if (jb.op == 0) {
      EncodeArgs a{jb.src, jb.dst, jb.L, jb.n, jb.t, 0};
      tile_encode(a, task.y, sm);
    } else {
      const uint8_t* loc = loc_tab + (size_t)jb.loc * kLocBytes;
      for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        s_er[i] = loc[i];
        s_lam[i] = loc[256 + i];
        s_ilp[i] = loc[512 + i];
      }
      __syncthreads();
      tile_recover(jb.dst, jb.L, jb.n, jb.e, pos_tab + jb.pos_off, task.y, sm, s_er, s_lam, s_ilp);
    }
    __syncthreads();
  }
}

}  // namespace

size_t batch_tiles(size_t L) { return (L + 32 * kCW - 1) / (32 * kCW); }

size_t batch_smem_bytes(int max_rows) { return (size_t)max_rows * kRowStride * 4; }

cudaError_t launch_batch(const BatchLaunch& b, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(b.counter, 0, sizeof(unsigned), s);
  if (e != cudaSuccess) return e;
  if (b.nrec > 0) {
    k_batch_locator<<<b.nrec, kThreads, 0, s>>>(b.jobs, b.rec_jobs, b.pos_tab, b.loc_tab);
    count_launches(1);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (b.ntasks == 0) return cudaSuccess;
  const size_t smem = batch_smem_bytes(b.max_rows);
  e = ensure_smem_attr(reinterpret_cast<const void*>(k_batch), smem);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch, kThreads, smem);
  if (e != cudaSuccess) return e;
  size_t grid = (size_t)sms * (size_t)std::max(per_sm, 1);
  if (grid > (size_t)b.ntasks) grid = (size_t)b.ntasks;
  k_batch<<<(unsigned)grid, kThreads, smem, s>>>(b.jobs, b.tasks, b.ntasks, b.counter, b.pos_tab, b.loc_tab);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace afrs
