// Smooth particle mesh Ewald on sm_100a: B-spline charge spreading, the
// influence-function convolution with the reciprocal energy and virial, and
// force / potential gathering; the 3D FFTs stay on cuFFT.
//
// Replaces MDIR's PME device stages (lib/Conversion/MDExecToGPU/
// DevicePME.cpp:38-75; PMEWeights.cpp, PMESpreadBricks.cpp, PMEConvolve.cpp,
// PMEGather.cpp; the fixed-point spreading of docs/pme.md, Section 3, D70)
// and its cuFFT entries (runtime/mdrt_cuda.c:2942-2990).  Equations as
// docs/pme.md, Sections 1 and 1.2: Q(k) = sum_i q_i M_p M_p M_p,
// E = 1/2 sum_m B(m) C(m) |F Q(m)|^2 with C = f/(pi V) exp(-pi^2 m^2/beta^2)/m^2,
// W_ab = sum_m E_m (delta_ab - 2 (1/m^2 + pi^2/beta^2) m_a m_b).
//
// B200 design: every stage reads the f32 frames of the places (the same
// array the pair kernel reads), so spreading and gathering walk atoms in the
// spatial order of the build and the grid lines they touch stay in L2 (a
// 64^3 grid is 1 MiB of a 126 MB L2).  Spreading uses `order` threads per
// atom, one per z point, each adding its order^2 products with f32
// reductions (or 64-bit integer reductions at 2^40 in the deterministic
// mode); the convolution scales the half-complex spectrum in place and sums
// energy and virial in f64 per block, summed again in a fixed order.
#include <cmath>
#include <cstdio>
#include <vector>

#include <type_traits>

#include "nb_context.h"
#include "nb_fft.cuh"
#include "nb_scan.cuh"
#include "nb_spline.cuh"

namespace {



template <int P, bool FIXED>
__global__ void __launch_bounds__(256) nb_spread(GridParams G, int64_t places,
                                                 const int32_t *__restrict__ sizes,
                                                 const int32_t *__restrict__ order,
                                                 const float4 *__restrict__ xq, float *__restrict__ grid,
                                                 unsigned long long *__restrict__ fixed, const int *halt) {
  if (halt && *halt) return;  // the MD step stopped at a stale list
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t p = t / P;
  int c = (int)(t - p * P);
  if (p >= places || p >= sizes[NB_SIZE_PLACES]) return;
  if (order[p] < 0) return;
  float4 v = xq[p];
  if (v.w == 0.f) return;
  int k0, k1, k2;
  float t0, t1, t2;
  nb_frac3(v, G, k0, k1, k2, t0, t1, t2);
  float w0[P], w1[P], w2[P];
  nb_bspline<P>(t0, w0, nullptr);
  nb_bspline<P>(t1, w1, nullptr);
  nb_bspline<P>(t2, w2, nullptr);
  int gz = k2 - c;
  if (gz < 0) gz += G.K2;
  float qz = v.w * nb_pick(w2, c);
#pragma unroll
  for (int jx = 0; jx < P; ++jx) {
    int gx = k0 - jx;
    if (gx < 0) gx += G.K0;
    float qxz = qz * w0[jx];
#pragma unroll
    for (int jy = 0; jy < P; ++jy) {
      int gy = k1 - jy;
      if (gy < 0) gy += G.K1;
      int64_t idx = ((int64_t)gx * G.K1 + gy) * G.K2 + gz;
      float val = qxz * w1[jy];
      if (FIXED)
        atomicAdd(fixed + idx, (unsigned long long)__double2ll_rn((double)val * NB_GRID_SCALE));
      else
        atomicAdd(grid + idx, val);
    }
  }
}

// ---------------------------------------------------------------------------
// The tiled spreading of large grids (MDIR D282, PMESpreadTile.cpp: bins of
// grid points, each bin's charges spread into a tile of shared memory, the
// tile added to the grid): fewer global atomics, each grid point hit by the
// tiles of at most 8 bins.  Here the places are binned by the tile of their
// first grid point (k0, k1, k2) / NB_TILE_EDGE, counted with one atomic a
// bin and warp (lanes of a bin found by match.any), the counts scanned, and
// the places scattered into bin order.  Mixed mode only: a tile sums its
// products in f32 in its own order, as MDIR's does.

__device__ __forceinline__ int nb_tile_of(int k0, int k1, int k2, int nb1, int nb2) {
  return ((k0 / NB_TILE_EDGE) * nb1 + k1 / NB_TILE_EDGE) * nb2 + k2 / NB_TILE_EDGE;
}

__global__ void __launch_bounds__(256) nb_tile_bin(GridParams G, int64_t places, const int32_t *__restrict__ sizes,
                                                  const int32_t *__restrict__ order, const float4 *__restrict__ xq,
                                                  int nb1, int nb2, int32_t *__restrict__ bin_of,
                                                  int32_t *__restrict__ rank_of, int32_t *__restrict__ count,
                                                  const int *halt) {
  if (halt && *halt) return;  // the MD step stopped at a stale list (every thread of the grid)
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int b = -1;
  if (p < places && p < sizes[NB_SIZE_PLACES] && order[p] >= 0) {
    float4 v = xq[p];
    if (v.w != 0.f) {
      int k0, k1, k2;
      float t0, t1, t2;
      nb_frac3(v, G, k0, k1, k2, t0, t1, t2);
      b = nb_tile_of(k0, k1, k2, nb1, nb2);
    }
  }
  // one count atomic for the lanes of a bin
  const unsigned FULL = 0xffffffffu;
  int lane = threadIdx.x & 31;
  unsigned peers = __match_any_sync(FULL, b);
  int leader = __ffs(peers) - 1;
  int base = 0;
  if (b >= 0 && lane == leader) base = atomicAdd(count + b, __popc(peers));
  base = __shfl_sync(FULL, base, leader);
  if (p < places) {
    bin_of[p] = b;
    rank_of[p] = base + __popc(peers & ((1u << lane) - 1u));
  }
}

__global__ void nb_tile_scatter(int64_t places, const int32_t *__restrict__ bin_of,
                                const int32_t *__restrict__ rank_of, const int32_t *__restrict__ start,
                                int32_t *__restrict__ sorted, const int *halt) {
  if (halt && *halt) return;
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= places) return;
  int b = bin_of[p];
  if (b >= 0) sorted[start[b] + rank_of[p]] = (int32_t)p;
}

// A block a bin: P threads a place (one z point each, as nb_spread) add the
// P^3 products into the tile of (NB_TILE_EDGE + P - 1)^3 points in shared
// memory, then the tile's nonzero points go to the grid.  A point that
// falls outside the tile (the binning's grid point not reproduced) goes to
// the grid directly.  The block empties its bin's count for the next
// binning.
template <int P>
__global__ void __launch_bounds__(128) nb_tile_spread(GridParams G, int nb1, int nb2,
                                                     const int32_t *__restrict__ start,
                                                     const int32_t *__restrict__ sorted,
                                                     const float4 *__restrict__ xq, float *__restrict__ grid,
                                                     int32_t *__restrict__ count, const int *halt) {
  constexpr int T = NB_TILE_EDGE + P - 1;
  __shared__ float tile[T * T * T];
  if (halt && *halt) return;
  const int b = blockIdx.x;
  for (int i = threadIdx.x; i < T * T * T; i += blockDim.x) tile[i] = 0.f;
  const int b2 = b % nb2, r = b / nb2, b1 = r % nb1, b0 = r / nb1;
  const int o0 = b0 * NB_TILE_EDGE - (P - 1), o1 = b1 * NB_TILE_EDGE - (P - 1), o2 = b2 * NB_TILE_EDGE - (P - 1);
  const int s0 = start[b], s1 = start[b + 1];
  __syncthreads();
  if (threadIdx.x == 0) count[b] = 0;
  for (int i = s0 * P + (int)threadIdx.x; i < s1 * P; i += blockDim.x) {
    int a = i / P, c = i - a * P;
    float4 v = xq[sorted[a]];
    int k0, k1, k2;
    float t0, t1, t2;
    nb_frac3(v, G, k0, k1, k2, t0, t1, t2);
    float w0[P], w1[P], w2[P];
    nb_bspline<P>(t0, w0, nullptr);
    nb_bspline<P>(t1, w1, nullptr);
    nb_bspline<P>(t2, w2, nullptr);
    float qz = v.w * nb_pick(w2, c);
    int lz = k2 - c - o2;
#pragma unroll
    for (int jx = 0; jx < P; ++jx) {
      int lx = k0 - jx - o0;
      float qxz = qz * w0[jx];
#pragma unroll
      for (int jy = 0; jy < P; ++jy) {
        int ly = k1 - jy - o1;
        float val = qxz * w1[jy];
        if ((unsigned)lx < (unsigned)T && (unsigned)ly < (unsigned)T && (unsigned)lz < (unsigned)T) {
          atomicAdd(&tile[(lx * T + ly) * T + lz], val);
        } else {
          int gx = k0 - jx, gy = k1 - jy, gz = k2 - c;
          if (gx < 0) gx += G.K0;
          if (gy < 0) gy += G.K1;
          if (gz < 0) gz += G.K2;
          atomicAdd(grid + ((int64_t)gx * G.K1 + gy) * G.K2 + gz, val);
        }
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < T * T * T; i += blockDim.x) {
    float val = tile[i];
    if (val == 0.f) continue;
    int lz = i % T, r2 = i / T, ly = r2 % T, lx = r2 / T;
    int gx = o0 + lx, gy = o1 + ly, gz = o2 + lz;
    // a tile reaches at most P - 1 points below 0 and at most NB_TILE_EDGE - 1
    // past the grid's last bin start: one wrap a side, for K >= T
    gx = gx < 0 ? gx + G.K0 : (gx >= G.K0 ? gx - G.K0 : gx);
    gy = gy < 0 ? gy + G.K1 : (gy >= G.K1 ? gy - G.K1 : gy);
    gz = gz < 0 ? gz + G.K2 : (gz >= G.K2 ? gz - G.K2 : gz);
    atomicAdd(grid + ((int64_t)gx * G.K1 + gy) * G.K2 + gz, val);
  }
}

// The fixed-point grid to f32, emptied behind: four points a thread with
// 16-byte loads and stores (the last total % 4 points one at a time).
__global__ void nb_fixed_to_grid(int64_t total, unsigned long long *__restrict__ fixed,
                                 float *__restrict__ grid) {
  int64_t k = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * 4;
  if (k + 4 <= total) {
    ulonglong2 a = *(const ulonglong2 *)(fixed + k), b = *(const ulonglong2 *)(fixed + k + 2);
    *(ulonglong2 *)(fixed + k) = make_ulonglong2(0ull, 0ull);
    *(ulonglong2 *)(fixed + k + 2) = make_ulonglong2(0ull, 0ull);
    *(float4 *)(grid + k) = make_float4((float)((double)(long long)a.x * (1.0 / NB_GRID_SCALE)),
                                        (float)((double)(long long)a.y * (1.0 / NB_GRID_SCALE)),
                                        (float)((double)(long long)b.x * (1.0 / NB_GRID_SCALE)),
                                        (float)((double)(long long)b.y * (1.0 / NB_GRID_SCALE)));
  } else {
    for (; k < total; ++k) {
      long long v = (long long)fixed[k];
      fixed[k] = 0ull;
      grid[k] = (float)((double)v * (1.0 / NB_GRID_SCALE));
    }
  }
}

struct ConvParams {
  int K0, K1, K2, H2;  // H2 = K2/2 + 1
  double L0, L1, L2;
  double h10 = 0.0, h20 = 0.0, h21 = 0.0;  // H^-1 (1,0), (2,0), (2,1) of a triclinic cell
  double pref;       // f / (pi V)
  double pi2_beta2;  // pi^2 / beta^2
};

// B C at half-complex point k: the B-spline moduli product times the Ewald
// reciprocal kernel f exp(-pi^2 m^2 / beta^2) / (pi V m^2); 0 at m = 0.
__device__ __forceinline__ double nb_bc(const ConvParams &C, const float *__restrict__ moduli, int64_t k,
                                        double &m0, double &m1, double &m2v, double &mm) {
  int i2 = (int)(k % C.H2);
  int64_t r = k / C.H2;
  int i1 = (int)(r % C.K1);
  int i0 = (int)(r / C.K1);
  // m = k0 a* + k1 b* + k2 c*, the reciprocal vectors the columns of H^-1
  double k0s = (i0 <= C.K0 / 2 ? i0 : i0 - C.K0), k1s = (i1 <= C.K1 / 2 ? i1 : i1 - C.K1);
  double k2s = (i2 <= C.K2 / 2 ? i2 : i2 - C.K2);
  m0 = k0s / C.L0;
  m1 = k1s / C.L1 + k0s * C.h10;
  m2v = k2s / C.L2 + k0s * C.h20 + k1s * C.h21;
  mm = m0 * m0 + m1 * m1 + m2v * m2v;
  if (k == 0) return 0.0;
  double B = (double)moduli[i0] * (double)moduli[C.K0 + i1] * (double)moduli[C.K0 + C.K1 + i2];
  return B * C.pref * exp(-C.pi2_beta2 * mm) / mm;
}

__global__ void nb_influence(ConvParams C, const float *__restrict__ moduli, float *__restrict__ out) {
  int64_t total = (int64_t)C.K0 * C.K1 * C.H2;
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= total) return;
  double m0, m1, m2v, mm;
  out[k] = (float)nb_bc(C, moduli, k, m0, m1, m2v, mm);
}

// The convolution of the MD step: the spectrum times the influence table
// (forces only, no energy sums).  With `grid`, it also empties the charge
// grid that the forward transform has read (total points), for the next
// step's spreading: no memset launch on the chain.
__global__ void nb_scale_spectrum(int64_t half, const float *__restrict__ influence, float2 *__restrict__ spec,
                                  float *__restrict__ grid, int64_t total, const int *halt) {
  if (halt && *halt) return;  // the MD step stopped at a stale list (it spread nothing either)
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (grid)
    for (int64_t i = k; i < total; i += half) grid[i] = 0.f;
  if (k >= half) return;
  float2 v = spec[k];
  float b = influence[k];
  spec[k] = make_float2(v.x * b, v.y * b);
}

// Multiplies the half-complex spectrum by B C and sums E and W in f64.
template <bool ENERGY>
__global__ void __launch_bounds__(256) nb_convolve(ConvParams C, const float *__restrict__ moduli,
                                                   float2 *__restrict__ spec,
                                                   double *__restrict__ partials) {
  __shared__ double s_part[8][7];
  int64_t total = (int64_t)C.K0 * C.K1 * C.H2;
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double v[7] = {0, 0, 0, 0, 0, 0, 0};
  if (k < total) {
    int i2 = (int)(k % C.H2);
    double m0, m1, m2v, mm;
    double bc = nb_bc(C, moduli, k, m0, m1, m2v, mm);
    float2 s = spec[k];
    spec[k] = make_float2((float)(s.x * bc), (float)(s.y * bc));
    if (ENERGY && k != 0) {
      double wgt = (i2 == 0 || (C.K2 % 2 == 0 && i2 == C.K2 / 2)) ? 1.0 : 2.0;
      double em = 0.5 * wgt * bc * ((double)s.x * s.x + (double)s.y * s.y);
      double f = -2.0 * (1.0 / mm + C.pi2_beta2);
      v[0] = em;
      v[1] = em * (1.0 + f * m0 * m0);
      v[2] = em * (1.0 + f * m1 * m1);
      v[3] = em * (1.0 + f * m2v * m2v);
      v[4] = em * f * m0 * m1;
      v[5] = em * f * m0 * m2v;
      v[6] = em * f * m1 * m2v;
    }
  }
  if (!ENERGY) return;
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
    for (int w = 0; w < 8; ++w) s += s_part[w][threadIdx.x];
    partials[(int64_t)blockIdx.x * 7 + threadIdx.x] = s;
  }
}

__global__ void nb_pme_sum(const double *__restrict__ partials, int nblocks, double *__restrict__ energy) {
  __shared__ double s[256][7];
  double v[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
    for (int k = 0; k < 7; ++k) v[k] += partials[(int64_t)b * 7 + k];
  for (int k = 0; k < 7; ++k) s[threadIdx.x][k] = v[k];
  __syncthreads();
  for (int stride = blockDim.x / 2; stride > 0; stride >>= 1) {
    if ((int)threadIdx.x < stride)
      for (int k = 0; k < 7; ++k) s[threadIdx.x][k] += s[threadIdx.x + stride][k];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    energy[NB_E_REC] = s[0][0];
    for (int k = 0; k < 6; ++k) energy[NB_W_REC + k] = s[0][1 + k];
  }
}

// ---------------------------------------------------------------------------
// The convolution on power-of-two grids in three kernels (nb_fft.cuh): the
// grid g[x][y][z] (z fastest) and the half-complex spectrum S[kx][ky][kz]
// (kz = 0..K2/2 fastest, cuFFT's R2C layout, so the influence table and the
// gathers are shared with the cuFFT chain).
//
//   nb_fft_planes_fwd   a block per x plane: rows y, y+1 go through one
//                       complex z transform as real and imaginary parts and
//                       are separated after it; the K2/2 + 1 z frequencies
//                       then take a y transform each, the real DC and
//                       Nyquist lines together as one complex line.  Empties
//                       the charge grid it read for the next spreading.
//   nb_fft_columns      a block per L columns (ky, kz): the x transform, the
//                       influence function B C (with the energy and virial
//                       sums when asked), the inverse x transform.
//   nb_fft_planes_inv   a block per x plane: the inverse y transforms, then
//                       the pairs of rows through one inverse z transform.
//
// Every array stays in L2 on the MD step's grid (1 MiB at 64^3).

template <int K>
__device__ __forceinline__ void nb_fft_load_tw(float2 *dst, const float2 *__restrict__ tw_all) {
  for (int i = threadIdx.x; i < K; i += blockDim.x) dst[i] = tw_all[nb_fft_tw_offset(K) + i];
}

// Shared memory of the plane kernels: twiddles, the row pairs S (lines of
// K2 + 1), the z frequencies T (lines of K1 + 1); lines rounded up to whole
// passes of the block's threads.
template <int K1, int K2>
struct NbFftPlane {
  static constexpr int H = K2 / 2, PR = K1 / 2;
  static constexpr int LA = NB_FFT_BLOCK / nb_fft_threads(K2), LB = NB_FFT_BLOCK / nb_fft_threads(K1);
  static constexpr int SL = (PR + LA - 1) / LA * LA, TL = (H + LB - 1) / LB * LB;
  static constexpr int S1 = K1 + 1, S2 = K2 + 1;
  static constexpr size_t bytes = sizeof(float2) * (size_t)(K1 + K2 + SL * S2 + TL * S1);
};

template <int K1, int K2, bool FIXED>
__global__ void __launch_bounds__(NB_FFT_BLOCK) nb_fft_planes_fwd(float *__restrict__ grid,
                                                                  unsigned long long *__restrict__ fixed,
                                                                  float2 *__restrict__ spec,
                                                                  const float2 *__restrict__ tw_all,
                                                                  const int *halt) {
  using Q = NbFftPlane<K1, K2>;
  constexpr int H = Q::H, S1 = Q::S1, S2 = Q::S2;
  extern __shared__ float2 nb_fft_sm[];
  float2 *tw1 = nb_fft_sm, *tw2 = tw1 + K1, *S = tw2 + K2, *T = S + Q::SL * S2;
  nb_fft_load_tw<K1>(tw1, tw_all);
  nb_fft_load_tw<K2>(tw2, tw_all);
  nb_grid_wait();
  const int stop = halt ? *halt : 0;  // the MD step stopped at a stale list
  const int tid = threadIdx.x;
  const int64_t plane = (int64_t)blockIdx.x * K1 * K2;
  // rows 2p and 2p + 1 as the real and imaginary parts of line p: every
  // load of a chunk in flight before the grid is emptied behind them
  constexpr int NA = Q::PR * K2 / NB_FFT_BLOCK, CH = NA < 8 ? NA : 8;
  static_assert(Q::PR * K2 % NB_FFT_BLOCK == 0, "whole rows per pass");
#pragma unroll 1
  for (int r0 = 0; r0 < NA; r0 += CH) {
    float va[CH], vb[CH];
#pragma unroll
    for (int r = 0; r < CH; ++r) {
      int i = tid + (r0 + r) * NB_FFT_BLOCK, p = i / K2, z = i - p * K2;
      int64_t a = plane + (int64_t)(2 * p) * K2 + z;
      if (FIXED) {
        va[r] = (float)((double)(long long)fixed[a] * (1.0 / NB_GRID_SCALE));
        vb[r] = (float)((double)(long long)fixed[a + K2] * (1.0 / NB_GRID_SCALE));
      } else {
        va[r] = grid[a];
        vb[r] = grid[a + K2];
      }
    }
    if (stop) return;
#pragma unroll
    for (int r = 0; r < CH; ++r) {
      int i = tid + (r0 + r) * NB_FFT_BLOCK, p = i / K2, z = i - p * K2;
      int64_t a = plane + (int64_t)(2 * p) * K2 + z;
      if (FIXED) {
        fixed[a] = 0ull;
        fixed[a + K2] = 0ull;
      } else {
        grid[a] = 0.f;
        grid[a + K2] = 0.f;
      }
      S[p * S2 + z] = make_float2(va[r], vb[r]);
    }
  }
  __syncthreads();
  {
    constexpr int TH = nb_fft_threads(K2);
    int g = tid / TH, t = tid - g * TH;
    for (int l = g; l < Q::SL; l += Q::LA) nb_fft_line<K2, false>(S + l * S2, t, tw2);
  }
  __syncthreads();
  // separate the pairs: A = (Z(k) + conj Z(K2-k))/2, B = (Z(k) - conj Z(K2-k))/2i;
  // line 0 of T holds DC + i Nyquist (both real) of each row
  for (int i = tid; i < Q::PR * H; i += NB_FFT_BLOCK) {
    int p = i / H, kz = i - p * H;
    float2 z = S[p * S2 + kz], a, b;
    if (kz == 0) {
      float2 nq = S[p * S2 + H];
      a = make_float2(z.x, nq.x);
      b = make_float2(z.y, nq.y);
    } else {
      float2 zc = S[p * S2 + K2 - kz];
      a = make_float2(0.5f * (z.x + zc.x), 0.5f * (z.y - zc.y));
      b = make_float2(0.5f * (z.y + zc.y), -0.5f * (z.x - zc.x));
    }
    T[kz * S1 + 2 * p] = a;
    T[kz * S1 + 2 * p + 1] = b;
  }
  __syncthreads();
  {
    constexpr int TH = nb_fft_threads(K1);
    int g = tid / TH, t = tid - g * TH;
    for (int l = g; l < Q::TL; l += Q::LB) nb_fft_line<K1, false>(T + l * S1, t, tw1);
  }
  __syncthreads();
  float2 *out = spec + (int64_t)blockIdx.x * K1 * (H + 1);
#pragma unroll 4
  for (int i = tid; i < K1 * (H + 1); i += NB_FFT_BLOCK) {
    int ky = i / (H + 1), kz = i - ky * (H + 1);
    float2 v;
    if (kz == 0 || kz == H) {
      // the two real lines out of their complex sum U = F0 + i FN
      float2 u = T[ky], w = T[(K1 - ky) & (K1 - 1)];
      v = kz == 0 ? make_float2(0.5f * (u.x + w.x), 0.5f * (u.y - w.y))
                  : make_float2(0.5f * (u.y + w.y), -0.5f * (u.x - w.x));
    } else {
      v = T[kz * S1 + ky];
    }
    out[i] = v;
  }
}

template <int K0>
struct NbFftColumns {
  static constexpr int L = NB_FFT_BLOCK / nb_fft_threads(K0), S0 = K0 + 1;
  static constexpr size_t bytes = sizeof(float2) * (size_t)(K0 + L * S0);
};

// ncols = K1 (K2/2 + 1) columns; block b takes columns b L .. b L + L - 1.
// Without ENERGY the spectrum is scaled by the f32 table `influence`; with
// it B C is formed in f64 per point as nb_convolve does and the block's
// energy and virial go to partials[7 b ..].
template <int K0, bool ENERGY>
__global__ void __launch_bounds__(NB_FFT_BLOCK) nb_fft_columns(int64_t ncols, float2 *__restrict__ spec,
                                                               const float *__restrict__ influence, ConvParams C,
                                                               const float *__restrict__ moduli,
                                                               double *__restrict__ partials,
                                                               const float2 *__restrict__ tw_all,
                                                               const int *halt) {
  using Q = NbFftColumns<K0>;
  constexpr int L = Q::L, S0 = Q::S0;
  extern __shared__ float2 nb_fft_sm[];
  float2 *tw = nb_fft_sm, *D = tw + K0;
  const int tid = threadIdx.x;
  const int64_t c0 = (int64_t)blockIdx.x * L;
  static_assert(K0 * L % NB_FFT_BLOCK == 0, "whole columns per pass");
  constexpr int NB = K0 * L / NB_FFT_BLOCK;  // 8: every load in flight at once
  // point r of this thread: kx = i / L, column c0 + i % L, i = tid + r NB_FFT_BLOCK
  float bc[NB];
  if (!ENERGY) {
    // the influence table is not written by the kernels before: read before the wait
#pragma unroll
    for (int r = 0; r < NB; ++r) {
      int i = tid + r * NB_FFT_BLOCK, kx = i / L, c = i - kx * L;
      bc[r] = c0 + c < ncols ? influence[(int64_t)kx * ncols + c0 + c] : 0.f;
    }
  }
  nb_fft_load_tw<K0>(tw, tw_all);
  nb_grid_wait();
  const int stop = halt ? *halt : 0;
  float2 v0[NB];
#pragma unroll
  for (int r = 0; r < NB; ++r) {
    int i = tid + r * NB_FFT_BLOCK, x = i / L, c = i - x * L;
    v0[r] = c0 + c < ncols ? spec[(int64_t)x * ncols + c0 + c] : make_float2(0.f, 0.f);
  }
  if (stop) return;
#pragma unroll
  for (int r = 0; r < NB; ++r) {
    int i = tid + r * NB_FFT_BLOCK, x = i / L, c = i - x * L;
    D[c * S0 + x] = v0[r];
  }
  __syncthreads();
  constexpr int TH = nb_fft_threads(K0);
  const int g = tid / TH, t = tid - g * TH;
  nb_fft_line<K0, false>(D + g * S0, t, tw);
  __syncthreads();
  double v[7] = {0, 0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int r = 0; r < NB; ++r) {
    int i = tid + r * NB_FFT_BLOCK, kx = i / L, c = i - kx * L;
    if (c0 + c >= ncols) continue;
    int64_t k = (int64_t)kx * ncols + c0 + c;
    float2 s = D[c * S0 + kx];
    if (ENERGY) {
      double m0, m1, m2v, mm;
      double b = nb_bc(C, moduli, k, m0, m1, m2v, mm);
      D[c * S0 + kx] = make_float2((float)(s.x * b), (float)(s.y * b));
      if (k != 0) {
        int i2 = (int)(k % C.H2);
        double wgt = (i2 == 0 || (C.K2 % 2 == 0 && i2 == C.K2 / 2)) ? 1.0 : 2.0;
        double em = 0.5 * wgt * b * ((double)s.x * s.x + (double)s.y * s.y);
        double f = -2.0 * (1.0 / mm + C.pi2_beta2);
        v[0] += em;
        v[1] += em * (1.0 + f * m0 * m0);
        v[2] += em * (1.0 + f * m1 * m1);
        v[3] += em * (1.0 + f * m2v * m2v);
        v[4] += em * f * m0 * m1;
        v[5] += em * f * m0 * m2v;
        v[6] += em * f * m1 * m2v;
      }
    } else {
      D[c * S0 + kx] = make_float2(s.x * bc[r], s.y * bc[r]);
    }
  }
  __syncthreads();
  nb_fft_line<K0, true>(D + g * S0, t, tw);
  __syncthreads();
#pragma unroll 4
  for (int i = tid; i < K0 * L; i += NB_FFT_BLOCK) {
    int x = i / L, c = i - x * L;
    if (c0 + c < ncols) spec[(int64_t)x * ncols + c0 + c] = D[c * S0 + x];
  }
  if (!ENERGY) return;
  __shared__ double s_part[NB_FFT_BLOCK / 32][7];
  int lane = tid & 31, warp = tid >> 5;
#pragma unroll
  for (int k = 0; k < 7; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  }
  if (lane == 0)
    for (int k = 0; k < 7; ++k) s_part[warp][k] = v[k];
  __syncthreads();
  if (tid < 7) {
    double s = 0.0;
    for (int w = 0; w < NB_FFT_BLOCK / 32; ++w) s += s_part[w][tid];
    partials[(int64_t)blockIdx.x * 7 + tid] = s;
  }
}

template <int K1, int K2>
__global__ void __launch_bounds__(NB_FFT_BLOCK) nb_fft_planes_inv(const float2 *__restrict__ spec,
                                                                  float *__restrict__ phi,
                                                                  const float2 *__restrict__ tw_all,
                                                                  const int *halt) {
  using Q = NbFftPlane<K1, K2>;
  constexpr int H = Q::H, S1 = Q::S1, S2 = Q::S2;
  extern __shared__ float2 nb_fft_sm[];
  float2 *tw1 = nb_fft_sm, *tw2 = tw1 + K1, *S = tw2 + K2, *T = S + Q::SL * S2;
  nb_fft_load_tw<K1>(tw1, tw_all);
  nb_fft_load_tw<K2>(tw2, tw_all);
  nb_grid_wait();
  const int stop = halt ? *halt : 0;
  const int tid = threadIdx.x;
  const float2 *in = spec + (int64_t)blockIdx.x * K1 * (H + 1);
  // the plane's spectrum, a chunk of loads in flight at a time
  constexpr int NC = (K1 * (H + 1) + NB_FFT_BLOCK - 1) / NB_FFT_BLOCK, CH = NC < 9 ? NC : 9;
#pragma unroll 1
  for (int r0 = 0; r0 < NC; r0 += CH) {
    float2 v[CH];
#pragma unroll
    for (int r = 0; r < CH; ++r) {
      int i = tid + (r0 + r) * NB_FFT_BLOCK;
      v[r] = i < K1 * (H + 1) ? in[i] : make_float2(0.f, 0.f);
    }
    if (stop) return;
#pragma unroll
    for (int r = 0; r < CH; ++r) {
      int i = tid + (r0 + r) * NB_FFT_BLOCK, ky = i / (H + 1), kz = i - ky * (H + 1);
      if (i < K1 * (H + 1) && kz != 0 && kz != H) T[kz * S1 + ky] = v[r];
    }
  }
  for (int ky = tid; ky < K1; ky += NB_FFT_BLOCK) {
    // the DC and Nyquist lines as one: F0 + i FN
    float2 f0 = in[ky * (H + 1)], fn = in[ky * (H + 1) + H];
    T[ky] = make_float2(f0.x - fn.y, f0.y + fn.x);
  }
  __syncthreads();
  {
    constexpr int TH = nb_fft_threads(K1);
    int g = tid / TH, t = tid - g * TH;
    for (int l = g; l < Q::TL; l += Q::LB) nb_fft_line<K1, true>(T + l * S1, t, tw1);
  }
  __syncthreads();
  // rows 2p, 2p + 1 as one line: Z(k) = A(k) + i B(k), Z(K2-k) = conj A(k) + i conj B(k)
  for (int i = tid; i < Q::PR * H; i += NB_FFT_BLOCK) {
    int p = i / H, kz = i - p * H;
    float2 a = T[kz * S1 + 2 * p], b = T[kz * S1 + 2 * p + 1];
    if (kz == 0) {
      S[p * S2] = make_float2(a.x, b.x);
      S[p * S2 + H] = make_float2(a.y, b.y);
    } else {
      S[p * S2 + kz] = make_float2(a.x - b.y, a.y + b.x);
      S[p * S2 + K2 - kz] = make_float2(a.x + b.y, b.x - a.y);
    }
  }
  __syncthreads();
  {
    constexpr int TH = nb_fft_threads(K2);
    int g = tid / TH, t = tid - g * TH;
    for (int l = g; l < Q::SL; l += Q::LA) nb_fft_line<K2, true>(S + l * S2, t, tw2);
  }
  __syncthreads();
  const int64_t plane = (int64_t)blockIdx.x * K1 * K2;
#pragma unroll 4
  for (int i = tid; i < Q::PR * K2; i += NB_FFT_BLOCK) {
    int p = i / K2, z = i - p * K2;
    float2 v = S[p * S2 + z];
    int64_t a = plane + (int64_t)(2 * p) * K2 + z;
    phi[a] = v.x;
    phi[a + K2] = v.y;
  }
}

// F_i = -q_i sum_k phi(k) grad(M M M); optional potential phi_i = sum_k phi(k) M M M.
template <int P>
__global__ void __launch_bounds__(128) nb_pme_gather(GridParams G, int64_t places,
                                                     const int32_t *__restrict__ sizes,
                                                     const int32_t *__restrict__ order,
                                                     const float4 *__restrict__ xq,
                                                     const float *__restrict__ phi,
                                                     float4 *__restrict__ out, float *__restrict__ pot) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= places || p >= sizes[NB_SIZE_PLACES]) return;
  if (order[p] < 0) {
    out[p] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (pot) pot[p] = 0.f;
    return;
  }
  float4 v = xq[p];
  int k0, k1, k2;
  float t0, t1, t2;
  nb_frac3(v, G, k0, k1, k2, t0, t1, t2);
  float w0[P], w1[P], w2[P], d0[P], d1[P], d2[P];
  nb_bspline<P>(t0, w0, d0);
  nb_bspline<P>(t1, w1, d1);
  nb_bspline<P>(t2, w2, d2);
  float g0 = 0.f, g1 = 0.f, g2 = 0.f, e = 0.f;
  int gzs[P];
#pragma unroll
  for (int jz = 0; jz < P; ++jz) {
    int gz = k2 - jz;
    gzs[jz] = gz < 0 ? gz + G.K2 : gz;
  }
#pragma unroll
  for (int jx = 0; jx < P; ++jx) {
    int gx = k0 - jx;
    if (gx < 0) gx += G.K0;
#pragma unroll
    for (int jy = 0; jy < P; ++jy) {
      int gy = k1 - jy;
      if (gy < 0) gy += G.K1;
      const float *row = phi + ((int64_t)gx * G.K1 + gy) * G.K2;
      float sz = 0.f, sdz = 0.f;
#pragma unroll
      for (int jz = 0; jz < P; ++jz) {
        float f = __ldg(row + gzs[jz]);
        sz = fmaf(f, w2[jz], sz);
        sdz = fmaf(f, d2[jz], sdz);
      }
      g0 = fmaf(d0[jx] * w1[jy], sz, g0);
      g1 = fmaf(w0[jx] * d1[jy], sz, g1);
      g2 = fmaf(w0[jx] * w1[jy], sdz, g2);
      e = fmaf(w0[jx] * w1[jy], sz, e);
    }
  }
  float q = v.w;
  float3 F = nb_frac_force(G, q, g0, g1, g2);
  out[p] = make_float4(F.x, F.y, F.z, 0.f);
  if (pot) pot[p] = e;
}

// The same gather with P threads per atom, one z point each (P a power of
// two dividing 32), summed over the P lanes by shuffles: four times the
// threads of a thread per atom, for a kernel that waits on L2 reads.
template <int P>
__global__ void __launch_bounds__(128) nb_pme_gather_split(GridParams G, int64_t places,
                                                           const int32_t *__restrict__ sizes,
                                                           const int32_t *__restrict__ order,
                                                           const float4 *__restrict__ xq,
                                                           const float *__restrict__ phi,
                                                           float4 *__restrict__ out, float *__restrict__ pot) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t p = t / P;
  int c = (int)(t & (P - 1));
  bool live = p < places && p < sizes[NB_SIZE_PLACES];
  bool atom = live && order[p] >= 0;
  float g0 = 0.f, g1 = 0.f, g2 = 0.f, e = 0.f;
  float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
  if (atom) {
    v = xq[p];
    int k0, k1, k2;
    float t0, t1, t2;
    nb_frac3(v, G, k0, k1, k2, t0, t1, t2);
    float w0[P], w1[P], w2[P], d0[P], d1[P], d2[P];
    nb_bspline<P>(t0, w0, d0);
    nb_bspline<P>(t1, w1, d1);
    nb_bspline<P>(t2, w2, d2);
    int gz = k2 - c;
    if (gz < 0) gz += G.K2;
    float wz = nb_pick(w2, c), dz = nb_pick(d2, c);
#pragma unroll
    for (int jx = 0; jx < P; ++jx) {
      int gx = k0 - jx;
      if (gx < 0) gx += G.K0;
#pragma unroll
      for (int jy = 0; jy < P; ++jy) {
        int gy = k1 - jy;
        if (gy < 0) gy += G.K1;
        float f = __ldg(phi + ((int64_t)gx * G.K1 + gy) * G.K2 + gz);
        float wxy = w0[jx] * w1[jy];
        g0 = fmaf(d0[jx] * w1[jy], f, g0);
        g1 = fmaf(w0[jx] * d1[jy], f, g1);
        e = fmaf(wxy, f, e);
        g2 = fmaf(wxy, f, g2);
      }
    }
    g0 *= wz;
    g1 *= wz;
    g2 *= dz;
    e *= wz;
  }
#pragma unroll
  for (int o = P / 2; o > 0; o >>= 1) {
    g0 += __shfl_xor_sync(0xffffffffu, g0, o);
    g1 += __shfl_xor_sync(0xffffffffu, g1, o);
    g2 += __shfl_xor_sync(0xffffffffu, g2, o);
    e += __shfl_xor_sync(0xffffffffu, e, o);
  }
  if (!live || c != 0) return;
  if (!atom) {
    out[p] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (pot) pot[p] = 0.f;
    return;
  }
  float q = v.w;
  float3 F = nb_frac_force(G, q, g0, g1, g2);
  out[p] = make_float4(F.x, F.y, F.z, 0.f);
  if (pot) pot[p] = e;
}

// The adjoint of the reciprocal forces for the force-matching product.
// With Q = sum_j q_j W_j, phi = Psi * Q and F_i = -q_i sum_k phi(k) grad W_i(k):
//   sum_i g_i . dF_i/dq_m = -g_m . sum_k phi(k) grad W_m(k) - sum_k W_m(k) psi(k),
//   psi = Psi * V,  V(k) = sum_i q_i g_i . grad W_i(k)   (Psi symmetric).
// nb_spread_dipole builds V; psi comes from the same FFTs and influence;
// nb_pme_adjoint_gather forms the two terms per atom.
template <int P>
__global__ void __launch_bounds__(256) nb_spread_dipole(GridParams G, int64_t places,
                                                        const int32_t *__restrict__ sizes,
                                                        const int32_t *__restrict__ order,
                                                        const float4 *__restrict__ xq, const float4 *__restrict__ gp,
                                                        float *__restrict__ grid) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t p = t / P;
  int c = (int)(t - p * P);
  if (p >= places || p >= sizes[NB_SIZE_PLACES]) return;
  if (order[p] < 0) return;
  float4 v = xq[p];
  float4 g = gp[p];
  if (v.w == 0.f) return;
  int k0, k1, k2;
  float t0, t1, t2;
  nb_frac(v.x, G.invL0, G.K0, k0, t0);
  nb_frac(v.y, G.invL1, G.K1, k1, t1);
  nb_frac(v.z, G.invL2, G.K2, k2, t2);
  float w0[P], w1[P], w2[P], d0[P], d1[P], d2[P];
  nb_bspline<P>(t0, w0, d0);
  nb_bspline<P>(t1, w1, d1);
  nb_bspline<P>(t2, w2, d2);
  float a0 = v.w * g.x * (float)G.K0 * G.invL0, a1 = v.w * g.y * (float)G.K1 * G.invL1,
        a2 = v.w * g.z * (float)G.K2 * G.invL2;
  int gz = k2 - c;
  if (gz < 0) gz += G.K2;
  float wz = nb_pick(w2, c), dz = nb_pick(d2, c);
#pragma unroll
  for (int jx = 0; jx < P; ++jx) {
    int gx = k0 - jx;
    if (gx < 0) gx += G.K0;
#pragma unroll
    for (int jy = 0; jy < P; ++jy) {
      int gy = k1 - jy;
      if (gy < 0) gy += G.K1;
      float val = (a0 * d0[jx] * w1[jy] + a1 * w0[jx] * d1[jy]) * wz + a2 * w0[jx] * w1[jy] * dz;
      atomicAdd(grid + ((int64_t)gx * G.K1 + gy) * G.K2 + gz, val);
    }
  }
}

// MODE 0: the two terms above; MODE 1: dE/dq_m = sum_k W_m(k) phi(k).
template <int P, int MODE>
__global__ void __launch_bounds__(128) nb_pme_adjoint_gather(GridParams G, int64_t places,
                                                             const int32_t *__restrict__ sizes,
                                                             const int32_t *__restrict__ order,
                                                             const float4 *__restrict__ xq,
                                                             const float4 *__restrict__ gp,
                                                             const float *__restrict__ phi,
                                                             const float *__restrict__ psi,
                                                             double *__restrict__ out) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= places || p >= sizes[NB_SIZE_PLACES]) return;
  if (order[p] < 0) return;
  float4 v = xq[p];
  float4 g = MODE == 0 ? gp[p] : make_float4(0.f, 0.f, 0.f, 0.f);
  int k0, k1, k2;
  float t0, t1, t2;
  nb_frac(v.x, G.invL0, G.K0, k0, t0);
  nb_frac(v.y, G.invL1, G.K1, k1, t1);
  nb_frac(v.z, G.invL2, G.K2, k2, t2);
  float w0[P], w1[P], w2[P], d0[P], d1[P], d2[P];
  nb_bspline<P>(t0, w0, d0);
  nb_bspline<P>(t1, w1, d1);
  nb_bspline<P>(t2, w2, d2);
  const float *sgrid = MODE == 0 ? psi : phi;
  double g0 = 0.0, g1 = 0.0, g2 = 0.0, s = 0.0;
  for (int jx = 0; jx < P; ++jx) {
    int gx = k0 - jx;
    if (gx < 0) gx += G.K0;
    for (int jy = 0; jy < P; ++jy) {
      int gy = k1 - jy;
      if (gy < 0) gy += G.K1;
      for (int jz = 0; jz < P; ++jz) {
        int gz = k2 - jz;
        if (gz < 0) gz += G.K2;
        int64_t idx = ((int64_t)gx * G.K1 + gy) * G.K2 + gz;
        double f = phi[idx], y = sgrid[idx];
        g0 += f * d0[jx] * w1[jy] * w2[jz];
        g1 += f * w0[jx] * d1[jy] * w2[jz];
        g2 += f * w0[jx] * w1[jy] * d2[jz];
        s += y * w0[jx] * w1[jy] * w2[jz];
      }
    }
  }
  if (MODE == 1) {
    out[p] += s;
    return;
  }
  double grad = g.x * g0 * G.K0 * G.invL0 + g.y * g1 * G.K1 * G.invL1 + g.z * g2 * G.K2 * G.invL2;
  out[p] += -grad - s;
}

// The same two terms with P threads per atom, one z point each (P a power
// of two dividing 32), in f32 partial sums over each thread's P x P points,
// summed over the P lanes by shuffles and added to the place's f64 value by
// its first lane.
template <int P, int MODE>
__global__ void __launch_bounds__(128) nb_pme_adjoint_gather_split(GridParams G, int64_t places,
                                                                   const int32_t *__restrict__ sizes,
                                                                   const int32_t *__restrict__ order,
                                                                   const float4 *__restrict__ xq,
                                                                   const float4 *__restrict__ gp,
                                                                   const float *__restrict__ phi,
                                                                   const float *__restrict__ psi,
                                                                   double *__restrict__ out) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t p = t / P;
  int c = (int)(t & (P - 1));
  bool live = p < places && p < sizes[NB_SIZE_PLACES];
  bool atom = live && order[p] >= 0;
  float g0 = 0.f, g1 = 0.f, g2 = 0.f, sv = 0.f;
  float4 g = make_float4(0.f, 0.f, 0.f, 0.f);
  if (atom) {
    float4 v = xq[p];
    if (MODE == 0) g = gp[p];
    int k0, k1, k2;
    float t0, t1, t2;
    nb_frac(v.x, G.invL0, G.K0, k0, t0);
    nb_frac(v.y, G.invL1, G.K1, k1, t1);
    nb_frac(v.z, G.invL2, G.K2, k2, t2);
    float w0[P], w1[P], w2[P], d0[P], d1[P], d2[P];
    nb_bspline<P>(t0, w0, d0);
    nb_bspline<P>(t1, w1, d1);
    nb_bspline<P>(t2, w2, d2);
    int gz = k2 - c;
    if (gz < 0) gz += G.K2;
    const float *sgrid = MODE == 0 ? psi : phi;
#pragma unroll
    for (int jx = 0; jx < P; ++jx) {
      int gx = k0 - jx;
      if (gx < 0) gx += G.K0;
#pragma unroll
      for (int jy = 0; jy < P; ++jy) {
        int gy = k1 - jy;
        if (gy < 0) gy += G.K1;
        int64_t idx = ((int64_t)gx * G.K1 + gy) * G.K2 + gz;
        float wxy = w0[jx] * w1[jy];
        sv = fmaf(wxy, __ldg(sgrid + idx), sv);
        if (MODE == 0) {
          float f = __ldg(phi + idx);
          g0 = fmaf(d0[jx] * w1[jy], f, g0);
          g1 = fmaf(w0[jx] * d1[jy], f, g1);
          g2 = fmaf(wxy, f, g2);
        }
      }
    }
    float wz = nb_pick(w2, c), dz = nb_pick(d2, c);
    g0 *= wz;
    g1 *= wz;
    g2 *= dz;
    sv *= wz;
  }
#pragma unroll
  for (int o = P / 2; o > 0; o >>= 1) {
    sv += __shfl_xor_sync(0xffffffffu, sv, o);
    if (MODE == 0) {
      g0 += __shfl_xor_sync(0xffffffffu, g0, o);
      g1 += __shfl_xor_sync(0xffffffffu, g1, o);
      g2 += __shfl_xor_sync(0xffffffffu, g2, o);
    }
  }
  if (!atom || c != 0) return;
  if (MODE == 1) {
    out[p] += (double)sv;
    return;
  }
  double grad = (double)g.x * g0 * G.K0 * G.invL0 + (double)g.y * g1 * G.K1 * G.invL1 +
                (double)g.z * g2 * G.K2 * G.invL2;
  out[p] += -grad - (double)sv;
}

inline int blocks_for(int64_t n, int t) { return (int)std::max<int64_t>(1, (n + t - 1) / t); }

// |b(m)|^2 of the SPME B-spline moduli along one edge, in f64 on the host.
std::vector<double> host_moduli(int K, int order) {
  std::vector<double> a(order + 1, 0.0), prev(order + 1, 0.0);
  // M_p at the integers 0..p-1 by the recursion with t = 0
  a[0] = 0.0;
  a[1] = 1.0;
  for (int m = 3; m <= order; ++m) {
    prev = a;
    for (int j = 0; j < m; ++j) {
      double left = j < m - 1 ? prev[j] : 0.0;
      double right = j > 0 ? prev[j - 1] : 0.0;
      a[j] = (j * left + (m - j) * right) / (m - 1);
    }
  }
  std::vector<double> out(K);
  for (int m = 0; m < K; ++m) {
    double re = 0.0, im = 0.0;
    for (int k = 0; k <= order - 2; ++k) {
      double arg = 2.0 * M_PI * m * k / K;
      re += a[k + 1] * cos(arg);
      im += a[k + 1] * sin(arg);
    }
    double s = re * re + im * im;
    out[m] = s < 1e-7 ? 0.0 : 1.0 / s;
  }
  for (int m = 0; m < K; ++m)
    if (out[m] == 0.0) out[m] = 0.5 * (out[(m + K - 1) % K] + out[(m + 1) % K]);
  return out;
}

// ---- host side of the three-kernel convolution -----------------------------

template <int K>
using NbK = std::integral_constant<int, K>;

bool nb_fft_size_ok(int k) { return k == 32 || k == 64 || k == 128; }

// f(NbK<K1>, NbK<K2>) for the plane sizes of the grid.
template <typename F>
bool nb_fft_planes(int k1, int k2, F &&f) {
#define NB_FFT_CASE(A, B)      \
  if (k1 == A && k2 == B) {    \
    f(NbK<A>(), NbK<B>());     \
    return true;               \
  }
  NB_FFT_CASE(32, 32) NB_FFT_CASE(32, 64) NB_FFT_CASE(32, 128)
  NB_FFT_CASE(64, 32) NB_FFT_CASE(64, 64) NB_FFT_CASE(64, 128)
  NB_FFT_CASE(128, 32) NB_FFT_CASE(128, 64) NB_FFT_CASE(128, 128)
#undef NB_FFT_CASE
  return false;
}

template <typename F>
bool nb_fft_column(int k0, F &&f) {
  if (k0 == 32) f(NbK<32>());
  else if (k0 == 64) f(NbK<64>());
  else if (k0 == 128) f(NbK<128>());
  else return false;
  return true;
}

template <typename Kern>
void nb_fft_smem(Kern kernel, size_t bytes) {
  if (bytes > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// The shared-memory opt-in of the kernels of a grid (once, at setup: not a
// stream operation, so not inside a captured step).
void nb_fft_prepare(const int K[3]) {
  nb_fft_planes(K[1], K[2], [](auto a, auto b) {
    constexpr int K1 = decltype(a)::value, K2 = decltype(b)::value;
    size_t bytes = NbFftPlane<K1, K2>::bytes;
    nb_fft_smem(nb_fft_planes_fwd<K1, K2, false>, bytes);
    nb_fft_smem(nb_fft_planes_fwd<K1, K2, true>, bytes);
    nb_fft_smem(nb_fft_planes_inv<K1, K2>, bytes);
  });
  nb_fft_column(K[0], [](auto a) {
    constexpr int K0 = decltype(a)::value;
    nb_fft_smem(nb_fft_columns<K0, false>, NbFftColumns<K0>::bytes);
    nb_fft_smem(nb_fft_columns<K0, true>, NbFftColumns<K0>::bytes);
  });
}

// Blocks of the column kernel on a grid.
int64_t nb_fft_column_blocks(const int K[3]) {
  int64_t ncols = (int64_t)K[1] * (K[2] / 2 + 1);
  int L = NB_FFT_BLOCK / nb_fft_threads(K[0]);
  return (ncols + L - 1) / L;
}

// The convolution of `grid` (or of the 2^40 fixed-point `fixed`, when
// non-null) into the potential `phi`, through `spec`; empties the grid it
// read.  energy: B C formed per point with the sums into partials (one
// block of seven per column block); else the table `influence`.  Launched
// chained after the spreading on s.
int nb_fft_convolve(const NbPme &P, float *grid, unsigned long long *fixed, float2 *spec, float *phi,
                    const float *influence, bool energy, const ConvParams &C, double *partials, const int *halt,
                    cudaStream_t s) {
  const int *K = P.K;
  const float2 *tw = P.fft_tw;
  int64_t ncols = (int64_t)K[1] * (K[2] / 2 + 1);
  cudaError_t e = cudaSuccess;
  bool ok = nb_fft_planes(K[1], K[2], [&](auto a, auto b) {
    constexpr int K1 = decltype(a)::value, K2 = decltype(b)::value;
    size_t bytes = NbFftPlane<K1, K2>::bytes;
    if (fixed)
      e = nb_launch_chained(nb_fft_planes_fwd<K1, K2, true>, dim3(K[0]), dim3(NB_FFT_BLOCK), bytes, s, grid, fixed,
                            spec, tw, halt);
    else
      e = nb_launch_chained(nb_fft_planes_fwd<K1, K2, false>, dim3(K[0]), dim3(NB_FFT_BLOCK), bytes, s, grid, fixed,
                            spec, tw, halt);
  });
  if (!ok || e != cudaSuccess) return -3;
  ok = nb_fft_column(K[0], [&](auto a) {
    constexpr int K0 = decltype(a)::value;
    dim3 blocks((unsigned)nb_fft_column_blocks(K));
    size_t bytes = NbFftColumns<K0>::bytes;
    if (energy)
      e = nb_launch_chained(nb_fft_columns<K0, true>, blocks, dim3(NB_FFT_BLOCK), bytes, s, ncols, spec, influence,
                            C, (const float *)P.moduli, partials, tw, halt);
    else
      e = nb_launch_chained(nb_fft_columns<K0, false>, blocks, dim3(NB_FFT_BLOCK), bytes, s, ncols, spec, influence,
                            C, (const float *)P.moduli, partials, tw, halt);
  });
  if (!ok || e != cudaSuccess) return -3;
  nb_fft_planes(K[1], K[2], [&](auto a, auto b) {
    constexpr int K1 = decltype(a)::value, K2 = decltype(b)::value;
    e = nb_launch_chained(nb_fft_planes_inv<K1, K2>, dim3(K[0]), dim3(NB_FFT_BLOCK), NbFftPlane<K1, K2>::bytes, s,
                          (const float2 *)spec, phi, tw, halt);
  });
  return e == cudaSuccess ? 0 : -3;
}

}  // namespace

// The spreading of the frames takes tiles when the tuning asks for them (the
// mixed mode; grids of at least a tile's edge).  MDIR tiles grids of
// 500,000 points and more by default (measured on an RTX 4090 and an RTX PRO
// 6000); on the B200 the global atomics were faster at 224^3 with 1.07 M
// atoms (a step of 2.22 ms with tiles against 2.08-2.16 ms), so the default
// keeps them.
bool nb_pme_tiled(const NbCtx &c) {
  const NbPme &P = c.pme;
  if (c.deterministic || c.pme_spread != 2 || !P.tile_count || !P.tile_bin) return false;
  if (P.order != 4 && P.order != 5 && P.order != 6 && P.order != 8) return false;
  // a tile wraps at most once a side: every K at least the tile's edge
  for (int a = 0; a < 3; ++a)
    if (P.K[a] < NB_TILE_EDGE + P.order - 1) return false;
  return true;
}

namespace {

// The frames' charges into `grid` (f32), or in the deterministic mode into
// the 2^40 fixed-point grid `fixed`; through tiles where nb_pme_tiled says.
void nb_spread_run(NbCtx &c, const GridParams &G, float *grid, unsigned long long *fixed, const int *halt,
                   cudaStream_t s) {
  NbPme &P = c.pme;
  if (nb_pme_tiled(c)) {
    int nb1 = P.tile_bins[1], nb2 = P.tile_bins[2];
    int nbins = P.tile_bins[0] * nb1 * nb2;
    nb_tile_bin<<<blocks_for(c.places_cap, 256), 256, 0, s>>>(G, c.places_cap, c.sizes, c.order, c.xq, nb1, nb2,
                                                               P.tile_bin, P.tile_rank, P.tile_count, halt);
    nb_scan(P.tile_count, P.tile_start, nbins, nullptr, P.tile_scratch, s);
    nb_tile_scatter<<<blocks_for(c.places_cap, 256), 256, 0, s>>>(c.places_cap, P.tile_bin, P.tile_rank,
                                                                   P.tile_start, P.tile_sorted, halt);
#define TILES(ORD)                                                                                    \
  nb_tile_spread<ORD><<<nbins, 128, 0, s>>>(G, nb1, nb2, P.tile_start, P.tile_sorted, c.xq, grid, \
                                            P.tile_count, halt)
    switch (P.order) {
      case 4: TILES(4); break;
      case 5: TILES(5); break;
      case 6: TILES(6); break;
      case 8: TILES(8); break;
    }
#undef TILES
    return;
  }
  int64_t threads = c.places_cap * P.order;
#define SPREAD(ORD)                                                                                      \
  if (c.deterministic)                                                                                   \
    nb_spread<ORD, true><<<blocks_for(threads, 256), 256, 0, s>>>(G, c.places_cap, c.sizes, c.order, c.xq, \
                                                                  grid, fixed, halt);                    \
  else                                                                                                   \
    nb_spread<ORD, false><<<blocks_for(threads, 256), 256, 0, s>>>(G, c.places_cap, c.sizes, c.order,      \
                                                                   c.xq, grid, fixed, halt);
  switch (P.order) {
    case 4: SPREAD(4); break;
    case 5: SPREAD(5); break;
    case 6: SPREAD(6); break;
    case 8: SPREAD(8); break;
  }
#undef SPREAD
}

}  // namespace

// The own transforms serve this context's grid (every K 32, 64 or 128) and
// are not switched off.
bool nb_fft_own(const NbCtx &c) { return c.pme.fft_tw != nullptr && c.pme_fft == 0; }

int nb_pme_setup(NbCtx &c, int k0, int k1, int k2, int order) {
  nb_pme_release(c);
  NbPme &P = c.pme;
  if (order != 4 && order != 5 && order != 6 && order != 8) return -2;
  P.K[0] = k0;
  P.K[1] = k1;
  P.K[2] = k2;
  P.order = order;
  int64_t total = (int64_t)k0 * k1 * k2;
  int64_t half = (int64_t)k0 * k1 * (k2 / 2 + 1);
  if (cudaMalloc(&P.grid, sizeof(float) * total) != cudaSuccess) return -1;
  if (cudaMalloc(&P.spec, sizeof(float2) * half) != cudaSuccess) return -1;
  if (cudaMalloc(&P.fixed, sizeof(unsigned long long) * total) != cudaSuccess) return -1;
  cudaMemset(P.fixed, 0, sizeof(unsigned long long) * total);
  if (cudaMalloc(&P.moduli, sizeof(float) * (k0 + k1 + k2)) != cudaSuccess) return -1;
  P.conv_blocks = blocks_for(half, 256);
  if (cudaMalloc(&P.partials, sizeof(double) * 7 * P.conv_blocks) != cudaSuccess) return -1;
  if (cudaMalloc(&P.influence, sizeof(float) * half) != cudaSuccess) return -1;
  for (double &k : P.infl_key) k = 0.0;
  std::vector<float> mod;
  for (int K : {k0, k1, k2}) {
    std::vector<double> m = host_moduli(K, order);
    for (double v : m) mod.push_back((float)v);
  }
  cudaMemcpy(P.moduli, mod.data(), sizeof(float) * mod.size(), cudaMemcpyHostToDevice);
  if (cufftPlan3d(&P.fwd, k0, k1, k2, CUFFT_R2C) != CUFFT_SUCCESS) return -3;
  if (cufftPlan3d(&P.bwd, k0, k1, k2, CUFFT_C2R) != CUFFT_SUCCESS) return -3;
  if (nb_fft_size_ok(k0) && nb_fft_size_ok(k1) && nb_fft_size_ok(k2)) {
    // e^(-2 pi i e/K) for K = 32, 64, 128, formed in f64
    std::vector<float2> tw(NB_FFT_TW_TOTAL);
    for (int K : {32, 64, 128})
      for (int e = 0; e < K; ++e) {
        double a = -2.0 * M_PI * (double)e / (double)K;
        tw[nb_fft_tw_offset(K) + e] = make_float2((float)std::cos(a), (float)std::sin(a));
      }
    if (cudaMalloc(&P.fft_tw, sizeof(float2) * NB_FFT_TW_TOTAL) != cudaSuccess) return -1;
    cudaMemcpy(P.fft_tw, tw.data(), sizeof(float2) * NB_FFT_TW_TOTAL, cudaMemcpyHostToDevice);
    nb_fft_prepare(P.K);
  }
  for (int a = 0; a < 3; ++a) P.tile_bins[a] = (P.K[a] + NB_TILE_EDGE - 1) / NB_TILE_EDGE;
  int64_t nbins = (int64_t)P.tile_bins[0] * P.tile_bins[1] * P.tile_bins[2];
  if (cudaMalloc(&P.tile_count, sizeof(int32_t) * (nbins + 1)) != cudaSuccess ||
      cudaMalloc(&P.tile_start, sizeof(int32_t) * (nbins + 1)) != cudaSuccess ||
      cudaMalloc(&P.tile_scratch, sizeof(int32_t) * (nbins / NB_SCAN_TILE + 64)) != cudaSuccess)
    return -1;
  cudaMemset(P.tile_count, 0, sizeof(int32_t) * (nbins + 1));
  if (c.places_cap > 0) {
    if (cudaMalloc(&P.pme_force, sizeof(float4) * c.places_cap) != cudaSuccess) return -1;
    if (cudaMalloc(&P.potential, sizeof(float) * c.places_cap) != cudaSuccess) return -1;
    if (cudaMalloc(&P.tile_bin, sizeof(int32_t) * c.places_cap) != cudaSuccess ||
        cudaMalloc(&P.tile_rank, sizeof(int32_t) * c.places_cap) != cudaSuccess ||
        cudaMalloc(&P.tile_sorted, sizeof(int32_t) * c.places_cap) != cudaSuccess)
      return -1;
  }
  P.on = true;
  return 0;
}

void nb_pme_release(NbCtx &c) {
  NbPme &P = c.pme;
  if (P.fwd) cufftDestroy(P.fwd);
  if (P.bwd) cufftDestroy(P.bwd);
  P.fwd = P.bwd = 0;
  for (void *p : {(void *)P.grid, (void *)P.spec, (void *)P.fixed, (void *)P.moduli,
                  (void *)P.pme_force, (void *)P.potential, (void *)P.partials, (void *)P.adj_grid,
                  (void *)P.influence, (void *)P.fft_tw, (void *)P.tile_count, (void *)P.tile_start,
                  (void *)P.tile_scratch, (void *)P.tile_bin, (void *)P.tile_rank, (void *)P.tile_sorted})
    if (p) cudaFree(p);
  P.fft_tw = nullptr;
  P.tile_count = P.tile_start = P.tile_scratch = nullptr;
  P.tile_bin = P.tile_rank = P.tile_sorted = nullptr;
  P.adj_grid = nullptr;
  P.influence = nullptr;
  P.grid = nullptr;
  P.spec = nullptr;
  P.fixed = nullptr;
  P.moduli = nullptr;
  P.pme_force = nullptr;
  P.potential = nullptr;
  P.partials = nullptr;
  P.on = false;
}

// The tilt terms of a triclinic cell (box = its diagonal, c.tilt = bx, cx,
// cy) for the fractions, the gradients and the reciprocal vectors: the
// entries of H^-1 below its diagonal, (1,0) = -bx/(ax by),
// (2,0) = (bx cy - by cx)/(ax by cz), (2,1) = -cy/(by cz).  Zero in an
// orthorhombic cell.
static void nb_cell_tilts(const NbCtx &c, const double box[3], GridParams &G, ConvParams *C) {
  double ax = box[0], by = box[1], cz = box[2], bx = c.tilt[0], cx = c.tilt[1], cy = c.tilt[2];
  double h10 = -bx / (ax * by), h20 = (bx * cy - by * cx) / (ax * by * cz), h21 = -cy / (by * cz);
  G.ta_b = (float)(bx / ax);
  G.ta_c = (float)(cx / ax);
  G.tb_c = (float)(cy / by);
  G.h10 = (float)h10;
  G.h20 = (float)h20;
  G.h21 = (float)h21;
  if (C) {
    C->h10 = h10;
    C->h20 = h20;
    C->h21 = h21;
  }
}

// The influence table of the context's cell for the convolutions that sum
// no energy (the forces, the adjoint), made again when the cell, the Ewald
// parameter, the Coulomb factor or the tilts change.
static int nb_pme_table(NbCtx &c, const double box[3], cudaStream_t s) {
  NbPme &P = c.pme;
  double key[8] = {box[0], box[1], box[2], c.beta, c.coulomb, c.tilt[0], c.tilt[1], c.tilt[2]};
  bool same = true;
  for (int k = 0; k < 8; ++k) same = same && key[k] == P.infl_key[k];
  if (same) return 0;
  if (nb_pme_influence(c, box, P.influence, s)) return -1;
  for (int k = 0; k < 8; ++k) P.infl_key[k] = key[k];
  return 0;
}

int nb_pme_run(NbCtx &c, const double box[3], bool energy, bool potential, cudaStream_t s) {
  NbPme &P = c.pme;
  if (!P.on) return 0;
  GridParams G;
  G.K0 = P.K[0];
  G.K1 = P.K[1];
  G.K2 = P.K[2];
  G.invL0 = (float)(1.0 / box[0]);
  G.invL1 = (float)(1.0 / box[1]);
  G.invL2 = (float)(1.0 / box[2]);
  nb_cell_tilts(c, box, G, nullptr);
  int64_t total = (int64_t)G.K0 * G.K1 * G.K2;
  int64_t half = (int64_t)G.K0 * G.K1 * (G.K2 / 2 + 1);
  if (!c.deterministic) cudaMemsetAsync(P.grid, 0, sizeof(float) * total, s);
  nb_spread_run(c, G, P.grid, P.fixed, nullptr, s);
  bool own = nb_fft_own(c);
  if (c.deterministic && !own) nb_fixed_to_grid<<<blocks_for((total + 3) / 4, 256), 256, 0, s>>>(total, P.fixed, P.grid);
  ConvParams C;
  C.K0 = G.K0;
  C.K1 = G.K1;
  C.K2 = G.K2;
  C.H2 = G.K2 / 2 + 1;
  C.L0 = box[0];
  C.L1 = box[1];
  C.L2 = box[2];
  C.pref = c.coulomb / (M_PI * box[0] * box[1] * box[2]);
  C.pi2_beta2 = M_PI * M_PI / (c.beta * c.beta);
  nb_cell_tilts(c, box, G, &C);
  if (own) {
    // spread grid -> potential in P.grid, the fixed-point grid read directly
    if (!energy && nb_pme_table(c, box, s)) return -1;
    if (nb_fft_convolve(P, P.grid, c.deterministic ? P.fixed : nullptr, P.spec, P.grid, P.influence, energy, C,
                        P.partials, nullptr, s))
      return -3;
    if (energy) nb_pme_sum<<<1, 256, 0, s>>>(P.partials, (int)nb_fft_column_blocks(P.K), c.energy);
  } else {
    cufftSetStream(P.fwd, s);
    cufftSetStream(P.bwd, s);
    if (cufftExecR2C(P.fwd, P.grid, (cufftComplex *)P.spec) != CUFFT_SUCCESS) return -3;
    if (energy) {
      nb_convolve<true><<<blocks_for(half, 256), 256, 0, s>>>(C, P.moduli, P.spec, P.partials);
      nb_pme_sum<<<1, 256, 0, s>>>(P.partials, P.conv_blocks, c.energy);
    } else {
      if (nb_pme_table(c, box, s)) return -1;
      nb_scale_spectrum<<<blocks_for(half, 256), 256, 0, s>>>(half, P.influence, P.spec, nullptr, 0, nullptr);
    }
    if (cufftExecC2R(P.bwd, (cufftComplex *)P.spec, P.grid) != CUFFT_SUCCESS) return -3;
  }
  float *pot = potential ? P.potential : nullptr;
  int blocks = blocks_for(c.places_cap, 128);
  float4 *pf = (float4 *)P.pme_force;
  switch (P.order) {
    case 4: nb_pme_gather_split<4><<<blocks_for(c.places_cap * 4, 128), 128, 0, s>>>(G, c.places_cap, c.sizes, c.order, c.xq, P.grid, pf, pot); break;
    case 5: nb_pme_gather<5><<<blocks, 128, 0, s>>>(G, c.places_cap, c.sizes, c.order, c.xq, P.grid, pf, pot); break;
    case 6: nb_pme_gather<6><<<blocks, 128, 0, s>>>(G, c.places_cap, c.sizes, c.order, c.xq, P.grid, pf, pot); break;
    case 8: nb_pme_gather_split<8><<<blocks_for(c.places_cap * 8, 128), 128, 0, s>>>(G, c.places_cap, c.sizes, c.order, c.xq, P.grid, pf, pot); break;
  }
  return 0;
}

// The reciprocal part of the parameter gradient in the charges, added per
// place into c.adj_q.  phi is recomputed by the forward stages (spread, FFT,
// influence, inverse FFT); in mode 0 the dipole grid V goes through the same
// FFT pair and influence to give psi.  The dipole spread uses f32 atomics
// in both modes of the forward (deterministic or not).
int nb_pme_adjoint_run(NbCtx &c, const double box[3], int mode, cudaStream_t s, const float *phi) {
  NbPme &P = c.pme;
  if (!P.on) return 0;
  GridParams G;
  G.K0 = P.K[0];
  G.K1 = P.K[1];
  G.K2 = P.K[2];
  G.invL0 = (float)(1.0 / box[0]);
  G.invL1 = (float)(1.0 / box[1]);
  G.invL2 = (float)(1.0 / box[2]);
  int64_t total = (int64_t)G.K0 * G.K1 * G.K2;
  int64_t half = (int64_t)G.K0 * G.K1 * (G.K2 / 2 + 1);
  if (!P.adj_grid && cudaMalloc(&P.adj_grid, sizeof(float) * total) != cudaSuccess) return -2;
  if (!phi) {
    int rc = nb_pme_run(c, box, false, false, s);  // phi in P.grid
    if (rc) return rc;
    phi = P.grid;
  }
  int blocks = blocks_for(c.places_cap, 128);
  if (mode == 1) {
    switch (P.order) {
      case 4: nb_pme_adjoint_gather_split<4, 1><<<blocks_for(c.places_cap * 4, 128), 128, 0, s>>>(G, c.places_cap, c.sizes, c.order, c.xq, nullptr, phi, nullptr, c.adj_q); break;
      case 5: nb_pme_adjoint_gather<5, 1><<<blocks, 128, 0, s>>>(G, c.places_cap, c.sizes, c.order, c.xq, nullptr, phi, nullptr, c.adj_q); break;
      case 6: nb_pme_adjoint_gather<6, 1><<<blocks, 128, 0, s>>>(G, c.places_cap, c.sizes, c.order, c.xq, nullptr, phi, nullptr, c.adj_q); break;
      case 8: nb_pme_adjoint_gather_split<8, 1><<<blocks_for(c.places_cap * 8, 128), 128, 0, s>>>(G, c.places_cap, c.sizes, c.order, c.xq, nullptr, phi, nullptr, c.adj_q); break;
    }
    return 0;
  }
  cudaMemsetAsync(P.adj_grid, 0, sizeof(float) * total, s);
  int64_t threads = c.places_cap * P.order;
  switch (P.order) {
    case 4: nb_spread_dipole<4><<<blocks_for(threads, 256), 256, 0, s>>>(G, c.places_cap, c.sizes, c.order, c.xq, c.adj_g, P.adj_grid); break;
    case 5: nb_spread_dipole<5><<<blocks_for(threads, 256), 256, 0, s>>>(G, c.places_cap, c.sizes, c.order, c.xq, c.adj_g, P.adj_grid); break;
    case 6: nb_spread_dipole<6><<<blocks_for(threads, 256), 256, 0, s>>>(G, c.places_cap, c.sizes, c.order, c.xq, c.adj_g, P.adj_grid); break;
    case 8: nb_spread_dipole<8><<<blocks_for(threads, 256), 256, 0, s>>>(G, c.places_cap, c.sizes, c.order, c.xq, c.adj_g, P.adj_grid); break;
  }
  ConvParams C;
  C.K0 = G.K0;
  C.K1 = G.K1;
  C.K2 = G.K2;
  C.H2 = G.K2 / 2 + 1;
  C.L0 = box[0];
  C.L1 = box[1];
  C.L2 = box[2];
  C.pref = c.coulomb / (M_PI * box[0] * box[1] * box[2]);
  C.pi2_beta2 = M_PI * M_PI / (c.beta * c.beta);
  if (nb_pme_table(c, box, s)) return -1;
  if (nb_fft_own(c)) {
    // V -> psi in place, three kernels
    if (nb_fft_convolve(P, P.adj_grid, nullptr, P.spec, P.adj_grid, P.influence, false, C, nullptr, nullptr, s))
      return -3;
  } else {
    // the plans run on this call's stream (a forward may have left them on another)
    cufftSetStream(P.fwd, s);
    cufftSetStream(P.bwd, s);
    if (cufftExecR2C(P.fwd, P.adj_grid, (cufftComplex *)P.spec) != CUFFT_SUCCESS) return -3;
    nb_scale_spectrum<<<blocks_for(half, 256), 256, 0, s>>>(half, P.influence, P.spec, nullptr, 0, nullptr);
    if (cufftExecC2R(P.bwd, (cufftComplex *)P.spec, P.adj_grid) != CUFFT_SUCCESS) return -3;
  }
  switch (P.order) {
    case 4: nb_pme_adjoint_gather_split<4, 0><<<blocks_for(c.places_cap * 4, 128), 128, 0, s>>>(G, c.places_cap, c.sizes, c.order, c.xq, c.adj_g, phi, P.adj_grid, c.adj_q); break;
    case 5: nb_pme_adjoint_gather<5, 0><<<blocks, 128, 0, s>>>(G, c.places_cap, c.sizes, c.order, c.xq, c.adj_g, phi, P.adj_grid, c.adj_q); break;
    case 6: nb_pme_adjoint_gather<6, 0><<<blocks, 128, 0, s>>>(G, c.places_cap, c.sizes, c.order, c.xq, c.adj_g, phi, P.adj_grid, c.adj_q); break;
    case 8: nb_pme_adjoint_gather_split<8, 0><<<blocks_for(c.places_cap * 8, 128), 128, 0, s>>>(G, c.places_cap, c.sizes, c.order, c.xq, c.adj_g, phi, P.adj_grid, c.adj_q); break;
  }
  return 0;
}

// ---------------------------------------------------------------------------
// PME over the frames of a batch (mdrtNbBatch).  The grids of the frames lie
// end to end, frames of one shape next to each other, so that one batched
// cuFFT plan pair per shape transforms them all; spreading, the influence
// function and gathering are one launch each, every atom or spectrum point
// reading its frame's grid, cell and moduli.

#include <algorithm>
#include <map>

namespace {

__device__ __forceinline__ GridParams nb_frame_grid(const NbFrameDev &F) {
  GridParams G;
  G.K0 = F.K0;
  G.K1 = F.K1;
  G.K2 = F.K2;
  G.invL0 = (float)(1.0 / F.L0);
  G.invL1 = (float)(1.0 / F.L1);
  G.invL2 = (float)(1.0 / F.L2);
  return G;
}

template <int P>
__global__ void __launch_bounds__(256) nb_batch_spread(int64_t places, const int32_t *__restrict__ sizes,
                                                       const int32_t *__restrict__ order,
                                                       const int32_t *__restrict__ atom_frame,
                                                       const NbFrameDev *__restrict__ frames,
                                                       const float4 *__restrict__ xq, float *__restrict__ grid) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t p = t / P;
  int c = (int)(t - p * P);
  if (p >= places || p >= sizes[NB_SIZE_PLACES]) return;
  int a = order[p];
  if (a < 0) return;
  float4 v = xq[p];
  if (v.w == 0.f) return;
  const NbFrameDev &F = frames[atom_frame[a]];
  GridParams G = nb_frame_grid(F);
  float *fg = grid + F.grid0;
  int k0, k1, k2;
  float t0, t1, t2;
  nb_frac(v.x, G.invL0, G.K0, k0, t0);
  nb_frac(v.y, G.invL1, G.K1, k1, t1);
  nb_frac(v.z, G.invL2, G.K2, k2, t2);
  float w0[P], w1[P], w2[P];
  nb_bspline<P>(t0, w0, nullptr);
  nb_bspline<P>(t1, w1, nullptr);
  nb_bspline<P>(t2, w2, nullptr);
  int gz = k2 - c;
  if (gz < 0) gz += G.K2;
  float qz = v.w * nb_pick(w2, c);
#pragma unroll
  for (int jx = 0; jx < P; ++jx) {
    int gx = k0 - jx;
    if (gx < 0) gx += G.K0;
    float qxz = qz * w0[jx];
#pragma unroll
    for (int jy = 0; jy < P; ++jy) {
      int gy = k1 - jy;
      if (gy < 0) gy += G.K1;
      atomicAdd(fg + ((int64_t)gx * G.K1 + gy) * G.K2 + gz, qxz * w1[jy]);
    }
  }
}

// Block b of the spectrum of frame f = blk_frame[b] (256 points of it).
template <bool ENERGY>
__global__ void __launch_bounds__(256) nb_batch_convolve(const int32_t *__restrict__ blk_frame,
                                                         const int32_t *__restrict__ blk0,
                                                         const NbFrameDev *__restrict__ frames,
                                                         const float *__restrict__ moduli, float2 *__restrict__ spec,
                                                         double *__restrict__ partials) {
  __shared__ double s_part[8][7];
  int f = blk_frame[blockIdx.x];
  const NbFrameDev &F = frames[f];
  int H2 = F.K2 / 2 + 1;
  int64_t total = (int64_t)F.K0 * F.K1 * H2;
  int64_t k = (int64_t)(blockIdx.x - blk0[f]) * blockDim.x + threadIdx.x;
  double v[7] = {0, 0, 0, 0, 0, 0, 0};
  if (k < total) {
    int i2 = (int)(k % H2);
    int64_t r = k / H2;
    int i1 = (int)(r % F.K1);
    int i0 = (int)(r / F.K1);
    double m0 = (i0 <= F.K0 / 2 ? i0 : i0 - F.K0) / F.L0;
    double m1 = (i1 <= F.K1 / 2 ? i1 : i1 - F.K1) / F.L1;
    double m2v = (i2 <= F.K2 / 2 ? i2 : i2 - F.K2) / F.L2;
    double mm = m0 * m0 + m1 * m1 + m2v * m2v;
    float2 *sp = spec + F.spec0;
    const float *md = moduli + F.mod0;
    float2 s = sp[k];
    double bc = 0.0;
    if (k != 0) {
      double B = (double)md[i0] * (double)md[F.K0 + i1] * (double)md[F.K0 + F.K1 + i2];
      bc = B * F.pref * exp(-F.pi2_beta2 * mm) / mm;
    }
    sp[k] = make_float2((float)(s.x * bc), (float)(s.y * bc));
    if (ENERGY && k != 0) {
      double wgt = (i2 == 0 || (F.K2 % 2 == 0 && i2 == F.K2 / 2)) ? 1.0 : 2.0;
      double em = 0.5 * wgt * bc * ((double)s.x * s.x + (double)s.y * s.y);
      double fm = -2.0 * (1.0 / mm + F.pi2_beta2);
      v[0] = em;
      v[1] = em * (1.0 + fm * m0 * m0);
      v[2] = em * (1.0 + fm * m1 * m1);
      v[3] = em * (1.0 + fm * m2v * m2v);
      v[4] = em * fm * m0 * m1;
      v[5] = em * fm * m0 * m2v;
      v[6] = em * fm * m1 * m2v;
    }
  }
  if (!ENERGY) return;
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
    for (int w = 0; w < 8; ++w) s += s_part[w][threadIdx.x];
    partials[(int64_t)blockIdx.x * 7 + threadIdx.x] = s;
  }
}

// P lanes an atom, one z point each (P a power of two dividing 32).
template <int P>
__global__ void __launch_bounds__(128) nb_batch_gather_split(int64_t places, const int32_t *__restrict__ sizes,
                                                             const int32_t *__restrict__ order,
                                                             const int32_t *__restrict__ atom_frame,
                                                             const NbFrameDev *__restrict__ frames,
                                                             const float4 *__restrict__ xq,
                                                             const float *__restrict__ grid,
                                                             float4 *__restrict__ out) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t p = t / P;
  int c = (int)(t & (P - 1));
  bool live = p < places && p < sizes[NB_SIZE_PLACES];
  int a = live ? order[p] : -1;
  float g0 = 0.f, g1 = 0.f, g2 = 0.f;
  float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
  GridParams G = {1, 1, 1, 1.f, 1.f, 1.f};
  if (a >= 0) {
    const NbFrameDev &F = frames[atom_frame[a]];
    G = nb_frame_grid(F);
    const float *phi = grid + F.grid0;
    v = xq[p];
    int k0, k1, k2;
    float t0, t1, t2;
    nb_frac(v.x, G.invL0, G.K0, k0, t0);
    nb_frac(v.y, G.invL1, G.K1, k1, t1);
    nb_frac(v.z, G.invL2, G.K2, k2, t2);
    float w0[P], w1[P], w2[P], d0[P], d1[P], d2[P];
    nb_bspline<P>(t0, w0, d0);
    nb_bspline<P>(t1, w1, d1);
    nb_bspline<P>(t2, w2, d2);
    int gz = k2 - c;
    if (gz < 0) gz += G.K2;
    float wz = nb_pick(w2, c), dz = nb_pick(d2, c);
#pragma unroll
    for (int jx = 0; jx < P; ++jx) {
      int gx = k0 - jx;
      if (gx < 0) gx += G.K0;
#pragma unroll
      for (int jy = 0; jy < P; ++jy) {
        int gy = k1 - jy;
        if (gy < 0) gy += G.K1;
        float f = __ldg(phi + ((int64_t)gx * G.K1 + gy) * G.K2 + gz);
        g0 = fmaf(d0[jx] * w1[jy], f, g0);
        g1 = fmaf(w0[jx] * d1[jy], f, g1);
        g2 = fmaf(w0[jx] * w1[jy], f, g2);
      }
    }
    g0 *= wz;
    g1 *= wz;
    g2 *= dz;
  }
#pragma unroll
  for (int o = P / 2; o > 0; o >>= 1) {
    g0 += __shfl_xor_sync(0xffffffffu, g0, o);
    g1 += __shfl_xor_sync(0xffffffffu, g1, o);
    g2 += __shfl_xor_sync(0xffffffffu, g2, o);
  }
  if (!live || c != 0) return;
  if (a < 0) {
    out[p] = make_float4(0.f, 0.f, 0.f, 0.f);
    return;
  }
  float q = v.w;
  float3 F = nb_frac_force(G, q, g0, g1, g2);
  out[p] = make_float4(F.x, F.y, F.z, 0.f);
}

}  // namespace

void nb_batch_pme_release(mdrtNbBatch &b) {
  for (auto &sh : b.shapes) {
    if (sh.fwd) cufftDestroy(sh.fwd);
    if (sh.bwd) cufftDestroy(sh.bwd);
  }
  b.shapes.clear();
  for (void *p : {(void *)b.conv_blk_frame, (void *)b.d_conv_blk0, (void *)b.conv_part})
    if (p) cudaFree(p);
  b.conv_blk_frame = nullptr;
  b.d_conv_blk0 = nullptr;
  b.conv_part = nullptr;
  b.conv_blocks = 0;
  b.pme = false;
  nb_pme_release(b.nb->c);
}

int nb_batch_pme_setup(mdrtNbBatch &b, const int32_t *grids, int order) {
  nb_batch_pme_release(b);
  if (order != 4 && order != 8) return -2;  // the split gather: a power of two dividing 32
  NbCtx &c = b.nb->c;
  NbPme &P = c.pme;
  // frames grouped by shape, in order of first appearance
  std::map<std::tuple<int, int, int>, std::vector<int>> by_shape;
  std::vector<std::tuple<int, int, int>> shape_order;
  for (int f = 0; f < b.frames; ++f) {
    auto key = std::make_tuple(grids[3 * f], grids[3 * f + 1], grids[3 * f + 2]);
    if (!by_shape.count(key)) shape_order.push_back(key);
    by_shape[key].push_back(f);
  }
  long long grid0 = 0, spec0 = 0;
  std::vector<float> mod;
  std::vector<int32_t> blk_frame, blk0(b.frames + 1, 0);
  std::vector<int> mod_of_shape;
  for (auto &key : shape_order) {
    int K0 = std::get<0>(key), K1 = std::get<1>(key), K2 = std::get<2>(key);
    int mod0 = (int)mod.size();
    for (int K : {K0, K1, K2}) {
      std::vector<double> m = host_moduli(K, order);
      for (double v : m) mod.push_back((float)v);
    }
    const std::vector<int> &fr = by_shape[key];
    mdrtNbBatch::Shape sh;
    sh.K[0] = K0;
    sh.K[1] = K1;
    sh.K[2] = K2;
    sh.count = (int)fr.size();
    sh.grid0 = grid0;
    sh.spec0 = spec0;
    sh.fwd = sh.bwd = 0;
    long long total = (long long)K0 * K1 * K2, half = (long long)K0 * K1 * (K2 / 2 + 1);
    for (int f : fr) {
      NbFrameDev &F = b.h_frames[f];
      F.K0 = K0;
      F.K1 = K1;
      F.K2 = K2;
      F.mod0 = mod0;
      F.grid0 = grid0;
      F.spec0 = spec0;
      grid0 += total;
      spec0 += half;
    }
    int n[3] = {K0, K1, K2};
    if (cufftPlanMany(&sh.fwd, 3, n, nullptr, 1, (int)total, nullptr, 1, (int)half, CUFFT_R2C, sh.count) !=
            CUFFT_SUCCESS ||
        cufftPlanMany(&sh.bwd, 3, n, nullptr, 1, (int)half, nullptr, 1, (int)total, CUFFT_C2R, sh.count) !=
            CUFFT_SUCCESS) {
      b.shapes.push_back(sh);
      return -3;
    }
    b.shapes.push_back(sh);
  }
  // the convolution's blocks, frame by frame
  for (int f = 0; f < b.frames; ++f) {
    const NbFrameDev &F = b.h_frames[f];
    long long half = (long long)F.K0 * F.K1 * (F.K2 / 2 + 1);
    int nb = (int)((half + 255) / 256);
    blk0[f] = (int)blk_frame.size();
    blk_frame.insert(blk_frame.end(), nb, f);
  }
  blk0[b.frames] = (int)blk_frame.size();
  b.conv_blocks = (int)blk_frame.size();
  b.h_conv_blk0 = blk0;
  if (cudaMalloc(&P.grid, sizeof(float) * std::max<long long>(grid0, 1)) != cudaSuccess ||
      cudaMalloc(&P.spec, sizeof(float2) * std::max<long long>(spec0, 1)) != cudaSuccess ||
      cudaMalloc(&P.moduli, sizeof(float) * mod.size()) != cudaSuccess ||
      cudaMalloc(&b.conv_part, sizeof(double) * 7 * std::max(b.conv_blocks, 1)) != cudaSuccess ||
      cudaMalloc(&b.conv_blk_frame, sizeof(int32_t) * std::max(b.conv_blocks, 1)) != cudaSuccess ||
      cudaMalloc(&b.d_conv_blk0, sizeof(int32_t) * (b.frames + 1)) != cudaSuccess)
    return -1;
  cudaMemcpy(P.moduli, mod.data(), sizeof(float) * mod.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(b.conv_blk_frame, blk_frame.data(), sizeof(int32_t) * b.conv_blocks, cudaMemcpyHostToDevice);
  cudaMemcpy(b.d_conv_blk0, blk0.data(), sizeof(int32_t) * (b.frames + 1), cudaMemcpyHostToDevice);
  b.grid_points = grid0;
  if (c.places_cap > 0) {
    if (cudaMalloc(&P.pme_force, sizeof(float4) * c.places_cap) != cudaSuccess) return -1;
    if (cudaMalloc(&P.potential, sizeof(float) * c.places_cap) != cudaSuccess) return -1;
  }
  P.order = order;
  P.on = true;
  b.order = order;
  b.pme = true;
  if (b.frames_dev)
    cudaMemcpy(b.frames_dev, b.h_frames.data(), sizeof(NbFrameDev) * b.frames, cudaMemcpyHostToDevice);
  return 0;
}

int nb_batch_pme_run(mdrtNbBatch &b, bool energy, cudaStream_t s) {
  NbCtx &c = b.nb->c;
  NbPme &P = c.pme;
  if (!b.pme || c.beta <= 0.0) return 0;
  cudaMemsetAsync(P.grid, 0, sizeof(float) * b.grid_points, s);
  int64_t threads = c.places_cap * b.order;
  if (b.order == 4)
    nb_batch_spread<4><<<blocks_for(threads, 256), 256, 0, s>>>(c.places_cap, c.sizes, c.order, b.atom_frame,
                                                               b.frames_dev, c.xq, P.grid);
  else
    nb_batch_spread<8><<<blocks_for(threads, 256), 256, 0, s>>>(c.places_cap, c.sizes, c.order, b.atom_frame,
                                                               b.frames_dev, c.xq, P.grid);
  for (auto &sh : b.shapes) {
    cufftSetStream(sh.fwd, s);
    if (cufftExecR2C(sh.fwd, P.grid + sh.grid0, (cufftComplex *)P.spec + sh.spec0) != CUFFT_SUCCESS) return -3;
  }
  if (energy)
    nb_batch_convolve<true><<<b.conv_blocks, 256, 0, s>>>(b.conv_blk_frame, b.d_conv_blk0, b.frames_dev, P.moduli,
                                                          P.spec, b.conv_part);
  else
    nb_batch_convolve<false><<<b.conv_blocks, 256, 0, s>>>(b.conv_blk_frame, b.d_conv_blk0, b.frames_dev, P.moduli,
                                                           P.spec, b.conv_part);
  for (auto &sh : b.shapes) {
    cufftSetStream(sh.bwd, s);
    if (cufftExecC2R(sh.bwd, (cufftComplex *)P.spec + sh.spec0, P.grid + sh.grid0) != CUFFT_SUCCESS) return -3;
  }
  float4 *pf = (float4 *)P.pme_force;
  if (b.order == 4)
    nb_batch_gather_split<4><<<blocks_for(c.places_cap * 4, 128), 128, 0, s>>>(
        c.places_cap, c.sizes, c.order, b.atom_frame, b.frames_dev, c.xq, P.grid, pf);
  else
    nb_batch_gather_split<8><<<blocks_for(c.places_cap * 8, 128), 128, 0, s>>>(
        c.places_cap, c.sizes, c.order, b.atom_frame, b.frames_dev, c.xq, P.grid, pf);
  return 0;
}

// The potential grid of the last force evaluation (K0 K1 K2 f32, in P.grid)
// to `out` (device), on s.
int nb_pme_potential_grid(NbCtx &c, float *out, cudaStream_t s) {
  NbPme &P = c.pme;
  if (!P.on) return -2;
  int64_t total = (int64_t)P.K[0] * P.K[1] * P.K[2];
  return cudaMemcpyAsync(out, P.grid, sizeof(float) * total, cudaMemcpyDeviceToDevice, s) == cudaSuccess ? 0 : -1;
}

// ---------------------------------------------------------------------------
// The reciprocal chain of the MD step when the update gathers (order 4): the
// integrator owns a charge grid (and its fixed-point form), a spectrum and a
// potential grid, so that force calls between runs leave them alone; the
// chain spreads the step's frames, transforms and applies the influence
// function, and the update gathers each atom's PME force from the potential.

int nb_pme_md_chain(NbCtx &c, const double box[3], float *qgrid, unsigned long long *qfixed, float2 *spec,
                    float *phi, const float *influence, const int *halt, cudaStream_t s) {
  NbPme &P = c.pme;
  GridParams G;
  G.K0 = P.K[0];
  G.K1 = P.K[1];
  G.K2 = P.K[2];
  G.invL0 = (float)(1.0 / box[0]);
  G.invL1 = (float)(1.0 / box[1]);
  G.invL2 = (float)(1.0 / box[2]);
  int64_t total = (int64_t)G.K0 * G.K1 * G.K2;
  int64_t half = (int64_t)G.K0 * G.K1 * (G.K2 / 2 + 1);
  nb_spread_run(c, G, qgrid, qfixed, halt, s);
  if (nb_fft_own(c)) {
    // the spread grid (empty before the spreading: this chain's forward
    // plane kernel empties it, or in the deterministic mode the fixed-point
    // grid, read directly) -> spectrum -> phi in three kernels
    ConvParams C{};
    return nb_fft_convolve(P, qgrid, c.deterministic ? qfixed : nullptr, spec, phi, influence, false, C, nullptr,
                           halt, s);
  }
  // the grid is empty: the conversion of the fixed-point grid empties that
  // one, the spectrum scaling of the last chain this one
  if (c.deterministic) nb_fixed_to_grid<<<blocks_for((total + 3) / 4, 256), 256, 0, s>>>(total, qfixed, qgrid);
  cufftSetStream(P.fwd, s);
  cufftSetStream(P.bwd, s);
  if (cufftExecR2C(P.fwd, qgrid, (cufftComplex *)spec) != CUFFT_SUCCESS) return -3;
  nb_scale_spectrum<<<blocks_for(half, 256), 256, 0, s>>>(half, influence, spec,
                                                          c.deterministic ? nullptr : qgrid, total, halt);
  if (cufftExecC2R(P.bwd, (cufftComplex *)spec, phi) != CUFFT_SUCCESS) return -3;
  return 0;
}

// The influence function B C of the cell `box` at every half-complex point,
// in f32 (the factor nb_convolve forms each time), for a chain that runs
// many times at one cell.
int nb_pme_influence(NbCtx &c, const double box[3], float *influence, cudaStream_t s) {
  NbPme &P = c.pme;
  ConvParams C;
  C.K0 = P.K[0];
  C.K1 = P.K[1];
  C.K2 = P.K[2];
  C.H2 = P.K[2] / 2 + 1;
  C.L0 = box[0];
  C.L1 = box[1];
  C.L2 = box[2];
  C.pref = c.coulomb / (M_PI * box[0] * box[1] * box[2]);
  C.pi2_beta2 = M_PI * M_PI / (c.beta * c.beta);
  GridParams G;
  nb_cell_tilts(c, box, G, &C);
  int64_t half = (int64_t)C.K0 * C.K1 * C.H2;
  nb_influence<<<blocks_for(half, 256), 256, 0, s>>>(C, P.moduli, influence);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
