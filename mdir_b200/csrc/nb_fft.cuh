// The transforms of the PME convolution on power-of-two grids (32, 64 or 128
// points a dimension), written for the reciprocal chain of the MD step so
// that a 3D transform pair is three kernels instead of cuFFT's six plus the
// influence launch between them.
//
// A K-point line lives in shared memory as K complex values.  N2 threads
// transform it as K = N1 x N2 (Cooley-Tukey, the "four-step" form): each
// thread takes the N1 points n2, n2 + N2, ... into registers and does an
// N1-point DFT, multiplies by the twiddles w_K^(n2 k1), and writes its row
// back; then each thread takes N1/N2 columns k1 and does N2-point DFTs over
// the rows, which leaves the spectrum in natural order.  The small DFTs are
// radix-2 decimation in frequency in registers.  Rows are written rotated
// by the thread's index, so that the eight threads of a line hit distinct
// shared-memory banks.
//
// Forward transforms use e^(-2 pi i nk/K) and inverse ones e^(+2 pi i nk/K);
// neither is normalized (cuFFT's convention, which the influence table and
// the gathers assume).
#pragma once
#include "nb_common.cuh"

// Threads of a block of the plane and column kernels.
#define NB_FFT_BLOCK 256

// Threads that transform one line of K points.
__host__ __device__ constexpr int nb_fft_threads(int K) { return K == 32 ? 4 : 8; }

// The bit reversal of i < R (R = 2, 4, 8 or 16): no recursion, so that it
// folds to a constant inside unrolled loops.
__host__ __device__ constexpr int nb_fft_brev(int i, int R) {
  return R == 16 ? ((i & 1) << 3) | ((i & 2) << 1) | ((i & 4) >> 1) | ((i & 8) >> 3)
       : R == 8  ? ((i & 1) << 2) | (i & 2) | ((i & 4) >> 2)
       : R == 4  ? ((i & 1) << 1) | ((i & 2) >> 1)
                 : i;
}

// v e^(-+2 pi i m/16): the multiples of an eighth turn in exact form, the
// others by the cosines of pi/8, pi/4 and 3 pi/8.
template <bool INV>
__device__ __forceinline__ float2 nb_fft_rot16(float2 v, int m) {
  constexpr float c1 = 0.92387953251128674f, c2 = 0.70710678118654752f, c3 = 0.38268343236508977f;
  m &= 15;
  if (m == 0) return v;
  if (m == 8) return make_float2(-v.x, -v.y);
  // the forward turn by -q quarter turns: (x, y) -> (y, -x); inverse (-y, x)
  if (m == 4) return INV ? make_float2(-v.y, v.x) : make_float2(v.y, -v.x);
  if (m == 12) return INV ? make_float2(v.y, -v.x) : make_float2(-v.y, v.x);
  if (m == 2 || m == 6 || m == 10 || m == 14) {
    // (cos, -+sin) of pi m/8 with |cos| = |sin| = c2
    float cs = (m == 2 || m == 14) ? c2 : -c2;
    float sn = (m == 2 || m == 6) ? c2 : -c2;
    if (!INV) sn = -sn;
    return make_float2(cs * v.x - sn * v.y, cs * v.y + sn * v.x);
  }
  // odd m: cos and sin of pi m/8 from c1 and c3
  const float cosv[8] = {1.f, c1, c2, c3, 0.f, -c3, -c2, -c1};
  float cs = m < 8 ? cosv[m] : cosv[16 - m];
  int ms = (m + 12) & 15;  // sin(x) = cos(x - pi/2)
  float sn = ms < 8 ? cosv[ms] : cosv[16 - ms];
  if (!INV) sn = -sn;
  return make_float2(cs * v.x - sn * v.y, cs * v.y + sn * v.x);
}

// An R-point DFT (R = 4, 8 or 16) of registers, in place, natural order.
template <int R, bool INV>
__device__ __forceinline__ void nb_fft_dft(float2 (&a)[R]) {
#pragma unroll
  for (int half = R / 2; half >= 1; half /= 2) {
#pragma unroll
    for (int base = 0; base < R; base += 2 * half) {
#pragma unroll
      for (int j = 0; j < half; ++j) {
        float2 u = a[base + j], v = a[base + j + half];
        a[base + j] = make_float2(u.x + v.x, u.y + v.y);
        a[base + j + half] = nb_fft_rot16<INV>(make_float2(u.x - v.x, u.y - v.y), j * (8 / half));
      }
    }
  }
  float2 b[R];
#pragma unroll
  for (int i = 0; i < R; ++i) b[nb_fft_brev(i, R)] = a[i];
#pragma unroll
  for (int i = 0; i < R; ++i) a[i] = b[i];
}

// The K-point transform of `line` (shared memory) by its N2 threads
// t = 0..N2-1, which must lie in one warp; every lane of the warp calls it
// (it synchronizes the warp).  tw[e] = e^(-2 pi i e/K), e < K.
template <int K, bool INV>
__device__ __forceinline__ void nb_fft_line(float2 *line, int t, const float2 *__restrict__ tw) {
  constexpr int N2 = nb_fft_threads(K), N1 = K / N2, J = N1 / N2;
  static_assert(N1 % N2 == 0, "the columns must split evenly over the threads");
  float2 a[N1];
#pragma unroll
  for (int n1 = 0; n1 < N1; ++n1) a[n1] = line[N2 * n1 + t];
  nb_fft_dft<N1, INV>(a);
#pragma unroll
  for (int k1 = 1; k1 < N1; ++k1) {
    float2 w = tw[t * k1];
    if (INV) w.y = -w.y;
    a[k1] = make_float2(a[k1].x * w.x - a[k1].y * w.y, a[k1].x * w.y + a[k1].y * w.x);
  }
  __syncwarp();
#pragma unroll
  for (int k1 = 0; k1 < N1; ++k1) line[t * N1 + ((k1 + t) & (N1 - 1))] = a[k1];
  __syncwarp();
  float2 b[J][N2];
#pragma unroll
  for (int j = 0; j < J; ++j) {
    int k1 = t + N2 * j;
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) b[j][n2] = line[n2 * N1 + ((k1 + n2) & (N1 - 1))];
  }
  __syncwarp();
#pragma unroll
  for (int j = 0; j < J; ++j) {
    nb_fft_dft<N2, INV>(b[j]);
    int k1 = t + N2 * j;
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) line[k1 + N1 * k2] = b[j][k2];
  }
}

// Offsets of the twiddle tables of K = 32, 64 and 128 in one array.
__host__ __device__ constexpr int nb_fft_tw_offset(int K) { return K == 32 ? 0 : K == 64 ? 32 : 96; }
#define NB_FFT_TW_TOTAL 224
