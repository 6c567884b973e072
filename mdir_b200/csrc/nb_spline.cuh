// Cardinal B-splines of smooth PME on the f32 frames of the places: the
// weights and slopes of an atom on the grid, and the grid point and fraction
// of a frame coordinate.  Shared by the PME kernels and the MD update (which
// gathers and spreads inside the step).
#pragma once
#include "nb_common.cuh"

// w[j] = M_p(t + j), dw[j] its slope, j = 0..p-1; weight j belongs to grid
// point floor(u) - j.  M_n(x) = (x M_{n-1}(x) + (n - x) M_{n-1}(x - 1))/(n - 1).
template <int P>
__device__ __forceinline__ void nb_bspline(float t, float *w, float *dw) {
  float a[P];
  a[0] = t;
  a[1] = 1.f - t;
#pragma unroll
  for (int j = 2; j < P; ++j) a[j] = 0.f;
#pragma unroll
  for (int m = 3; m <= P; ++m) {
    float prev[P];
#pragma unroll
    for (int j = 0; j < P; ++j) prev[j] = a[j];
    if (m == P && dw) {
#pragma unroll
      for (int j = 0; j < P; ++j) dw[j] = (j < m - 1 ? prev[j] : 0.f) - (j > 0 ? prev[j - 1] : 0.f);
    }
    float inv = 1.f / (float)(m - 1);
#pragma unroll
    for (int j = 0; j < P; ++j) {
      if (j < m) {
        float left = j < m - 1 ? prev[j] : 0.f;
        float right = j > 0 ? prev[j - 1] : 0.f;
        a[j] = ((t + j) * left + ((float)m - t - j) * right) * inv;
      }
    }
  }
  if (P == 2 && dw) {
    dw[0] = 1.f;
    dw[1] = -1.f;
  }
#pragma unroll
  for (int j = 0; j < P; ++j) w[j] = a[j];
}

// The grid point and fraction of a frame coordinate x (centred on the
// cell: the fractional coordinate is x / L + 1/2).
__device__ __forceinline__ void nb_frac(float x, float invL, int K, int &k0, float &t) {
  float f = fmaf(x, invL, 0.5f);
  f -= floorf(f);
  float u = f * (float)K;
  float fl = floorf(u);
  int k = (int)fl;
  if (k >= K) k -= K;
  if (k < 0) k += K;
  k0 = k;
  t = u - fl;
  if (t >= 1.f) t = 0.f;
}

struct GridParams {
  int K0, K1, K2;
  float invL0, invL1, invL2;
};
