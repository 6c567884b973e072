// Exclusive scan of int32 counts on the device, in three launches that do
// not depend on the data (so that they can be captured in a CUDA graph):
// block sums of 4096 elements, one block scanning up to 4096 block sums,
// and the final pass.  out[n] receives the total.  Capacity: 16.7M inputs.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#define NB_SCAN_THREADS 1024
#define NB_SCAN_PER_THREAD 4
#define NB_SCAN_TILE (NB_SCAN_THREADS * NB_SCAN_PER_THREAD)

// Internal to each file that includes it (the build and the tiled PME
// spreading both scan).
namespace {

__device__ __forceinline__ int nb_block_exclusive_scan(int v, int *smem_warp, int &total) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) smem_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int nw = blockDim.x >> 5;
    int w = lane < nw ? smem_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    smem_warp[lane] = w;
  }
  __syncthreads();
  int before = warp > 0 ? smem_warp[warp - 1] : 0;
  total = smem_warp[(blockDim.x >> 5) - 1];
  __syncthreads();
  return before + x - v;
}

__global__ void nb_scan_blocks(const int *__restrict__ in, const int *__restrict__ n_ptr, int n_static,
                               int *__restrict__ block_sums) {
  __shared__ int sw[32];
  int n = n_ptr ? *n_ptr : n_static;
  int64_t base = (int64_t)blockIdx.x * NB_SCAN_TILE + threadIdx.x * NB_SCAN_PER_THREAD;
  int s = 0;
#pragma unroll
  for (int k = 0; k < NB_SCAN_PER_THREAD; ++k)
    if (base + k < n) s += in[base + k];
  int total;
  nb_block_exclusive_scan(s, sw, total);
  if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

__global__ void nb_scan_sums(int *__restrict__ block_sums, int nblocks) {
  __shared__ int sw[32];
  int base = threadIdx.x * NB_SCAN_PER_THREAD;
  int v[NB_SCAN_PER_THREAD];
  int s = 0;
#pragma unroll
  for (int k = 0; k < NB_SCAN_PER_THREAD; ++k) {
    v[k] = base + k < nblocks ? block_sums[base + k] : 0;
    s += v[k];
  }
  int total;
  int ex = nb_block_exclusive_scan(s, sw, total);
#pragma unroll
  for (int k = 0; k < NB_SCAN_PER_THREAD; ++k) {
    if (base + k < nblocks) block_sums[base + k] = ex;
    ex += v[k];
  }
  if (threadIdx.x == 0) block_sums[nblocks] = total;
}

__global__ void nb_scan_final(const int *__restrict__ in, const int *__restrict__ n_ptr, int n_static,
                              const int *__restrict__ block_sums, int nblocks, int *__restrict__ out) {
  __shared__ int sw[32];
  int n = n_ptr ? *n_ptr : n_static;
  int64_t base = (int64_t)blockIdx.x * NB_SCAN_TILE + threadIdx.x * NB_SCAN_PER_THREAD;
  int v[NB_SCAN_PER_THREAD];
  int s = 0;
#pragma unroll
  for (int k = 0; k < NB_SCAN_PER_THREAD; ++k) {
    v[k] = base + k < n ? in[base + k] : 0;
    s += v[k];
  }
  int total;
  int ex = nb_block_exclusive_scan(s, sw, total) + block_sums[blockIdx.x];
#pragma unroll
  for (int k = 0; k < NB_SCAN_PER_THREAD; ++k) {
    if (base + k < n) out[base + k] = ex;
    ex += v[k];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = block_sums[nblocks];
}

// Scans in[0..n) into out[0..n] (exclusive, out[n] = total).  n_max bounds
// n (the grid is sized by it); n_ptr, if not null, holds the actual n on
// the device.  scratch holds at least n_max / NB_SCAN_TILE + 2 ints.
inline void nb_scan(const int *in, int *out, int n_max, const int *n_ptr, int *scratch,
                    cudaStream_t stream) {
  int nblocks = (n_max + NB_SCAN_TILE - 1) / NB_SCAN_TILE;
  if (nblocks < 1) nblocks = 1;
  nb_scan_blocks<<<nblocks, NB_SCAN_THREADS, 0, stream>>>(in, n_ptr, n_max, scratch);
  nb_scan_sums<<<1, NB_SCAN_THREADS, 0, stream>>>(scratch, nblocks);
  nb_scan_final<<<nblocks, NB_SCAN_THREADS, 0, stream>>>(in, n_ptr, n_max, scratch, nblocks, out);
}

}  // namespace
