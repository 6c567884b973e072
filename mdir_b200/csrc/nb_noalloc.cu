// mdrtNbExcludedNoAlloc: the excluded-pair Ewald correction with no device
// allocation at all, for callers that cannot allocate.
//
// Who needs it: a host program that owns all device memory through its own
// fixed pool and forbids any other allocation, a plugin loaded into such a
// program, or a real-time loop that must not pay the device-wide
// synchronization that cudaFree implies.  The regular path (mdrtNbForce)
// keeps its per-block partial sums in buffers that the context allocates;
// this variant keeps them in a file-scope __device__ array instead, so that
// the caller provides only inputs and outputs.
//
// The array holds the partials of at most MDRT_NB_NOALLOC_MAX_PAIRS pairs
// (256 pairs a block, 8 doubles a block: 256 KiB).  Every GPU that loads this
// library holds it until the process exits.  Every call shares it and it
// keeps the last call's contents; each call overwrites the partials of its
// own blocks before its reduction reads them, so nothing needs clearing, but
// two calls that overlap on the GPU (on different streams) race on it.
#include <cmath>
#include <cstdio>
#include <mutex>

#include "../../include/mdrt_nb.h"

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = (MDRT_NB_NOALLOC_MAX_PAIRS + kThreads - 1) / kThreads;
constexpr int kMaxDevices = 64;

// The scratch: per-block partial sums (energy, six virial entries, pad).
static __device__ __align__(256) double g_excl_partials[kMaxBlocks * 8];

// Its device address, found once per device (the host-side name of a
// __device__ array is not a device address) and kept for the life of the
// process: after a cudaDeviceReset the kept address may be stale, so a
// program that resets a device does not call this entry point on it again.
std::mutex g_mutex;
double *g_partials[kMaxDevices] = {nullptr};

int scratch_on_current_device(double **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return MDRT_NB_CUDA_ERROR;
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_partials[dev]) {
    double *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void **)&p, g_excl_partials);
    if (e != cudaSuccess) {
      fprintf(stderr, "mdrt_nb: cudaGetSymbolAddress of the scratch of mdrtNbExcludedNoAlloc: %s\n",
              cudaGetErrorString(e));
      return MDRT_NB_CUDA_ERROR;
    }
    g_partials[dev] = p;
  }
  *out = g_partials[dev];
  return MDRT_NB_OK;
}

// -f q_i q_j erf(beta r)/r over the pairs (i < j) in the minimum image, in
// f64 from the f64 positions; forces added with f64 atomics; the energy and
// virial of each block to the scratch.
__global__ void __launch_bounds__(kThreads) excluded_noalloc(int64_t npairs, const int32_t *__restrict__ pairs,
                                                             const double *__restrict__ x,
                                                             const double *__restrict__ q, double Lx, double Ly,
                                                             double Lz, double beta, double coulomb,
                                                             double *__restrict__ forces, double *partials) {
  __shared__ double s_part[kThreads / 32][8];
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (k < npairs) {
    int i = pairs[2 * k], j = pairs[2 * k + 1];
    double d0 = x[3 * i] - x[3 * j], d1 = x[3 * i + 1] - x[3 * j + 1], d2 = x[3 * i + 2] - x[3 * j + 2];
    d0 -= Lx * rint(d0 / Lx);
    d1 -= Ly * rint(d1 / Ly);
    d2 -= Lz * rint(d2 / Lz);
    double r2 = d0 * d0 + d1 * d1 + d2 * d2;
    double qq = coulomb * q[i] * q[j];
    if (qq != 0.0 && r2 > 0.0) {
      double r = sqrt(r2);
      double ef = erf(beta * r);
      double g = 2.0 * beta / sqrt(M_PI) * exp(-beta * beta * r2);
      double fs = qq * (g / r2 - ef / (r2 * r));
      atomicAdd(forces + 3 * i, fs * d0);
      atomicAdd(forces + 3 * i + 1, fs * d1);
      atomicAdd(forces + 3 * i + 2, fs * d2);
      atomicAdd(forces + 3 * j, -fs * d0);
      atomicAdd(forces + 3 * j + 1, -fs * d1);
      atomicAdd(forces + 3 * j + 2, -fs * d2);
      v[0] = -qq * ef / r;
      v[1] = d0 * fs * d0;
      v[2] = d1 * fs * d1;
      v[3] = d2 * fs * d2;
      v[4] = d0 * fs * d1;
      v[5] = d0 * fs * d2;
      v[6] = d1 * fs * d2;
    }
  }
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < 7; ++c) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[c] += __shfl_xor_sync(0xffffffffu, v[c], o);
  }
  if (lane == 0)
    for (int c = 0; c < 7; ++c) s_part[warp][c] = v[c];
  __syncthreads();
  if (threadIdx.x < 7) {
    double s = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) s += s_part[w][threadIdx.x];
    partials[(int64_t)blockIdx.x * 8 + threadIdx.x] = s;
  }
}

// The partials of `nblocks` blocks summed in a fixed order into out[7].
__global__ void excluded_noalloc_sum(const double *partials, int nblocks, double *out) {
  __shared__ double s[kThreads][7];
  double v[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
    for (int c = 0; c < 7; ++c) v[c] += partials[(int64_t)b * 8 + c];
  for (int c = 0; c < 7; ++c) s[threadIdx.x][c] = v[c];
  __syncthreads();
  for (int stride = blockDim.x / 2; stride > 0; stride >>= 1) {
    if ((int)threadIdx.x < stride)
      for (int c = 0; c < 7; ++c) s[threadIdx.x][c] += s[threadIdx.x + stride][c];
    __syncthreads();
  }
  if (threadIdx.x < 7) out[threadIdx.x] = s[0][threadIdx.x];
}

}  // namespace

extern "C" int32_t mdrtNbExcludedNoAlloc(const double *x, const double *charges, const int32_t *pairs,
                                         int64_t npairs, const double box[3], double beta, double coulomb,
                                         double *forces, double *energy_virial, void *stream) {
  if (!x || !charges || !forces || !energy_virial || !box || npairs < 0 || (npairs > 0 && !pairs))
    return MDRT_NB_INVALID_ARGUMENT;
  if (npairs > MDRT_NB_NOALLOC_MAX_PAIRS) {
    fprintf(stderr,
            "mdrt_nb: mdrtNbExcludedNoAlloc: %lld excluded pairs exceed its fixed scratch of %d pairs; "
            "use mdrtNbForce, which allocates\n",
            (long long)npairs, MDRT_NB_NOALLOC_MAX_PAIRS);
    return MDRT_NB_INVALID_ARGUMENT;
  }
  for (int k = 0; k < 3; ++k)
    if (!(box[k] > 0.0) || !std::isfinite(box[k])) return MDRT_NB_INVALID_BOX;
  double *partials = nullptr;
  int32_t s = scratch_on_current_device(&partials);
  if (s) return s;
  cudaStream_t st = (cudaStream_t)stream;
  int blocks = (int)((npairs + kThreads - 1) / kThreads);
  if (blocks > 0)
    excluded_noalloc<<<blocks, kThreads, 0, st>>>(npairs, pairs, x, charges, box[0], box[1], box[2], beta, coulomb,
                                                  forces, partials);
  excluded_noalloc_sum<<<1, kThreads, 0, st>>>(partials, blocks, energy_virial);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "mdrt_nb: mdrtNbExcludedNoAlloc: %s\n", cudaGetErrorString(e));
    return MDRT_NB_CUDA_ERROR;
  }
  return MDRT_NB_OK;
}
