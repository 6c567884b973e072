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
  // a triclinic cell (0 in an orthorhombic one): the fractions' tilt terms
  // bx/ax, cx/ax, cy/by, and the off-diagonal entries (1,0), (2,0), (2,1)
  // of H^-1, which take the spline slopes to Cartesian gradients
  float ta_b = 0.f, ta_c = 0.f, tb_c = 0.f;
  float h10 = 0.f, h20 = 0.f, h21 = 0.f;
};

// The grid points and fractions of a centred frame v in a triclinic cell
// (the position p = v + diag/2 = fa a + fb b + fc c): fc = v.z/cz + 1/2,
// fb = v.y/by + 1/2 - fc cy/by, fa = v.x/ax + 1/2 - fb bx/ax - fc cx/ax; in
// an orthorhombic cell these are nb_frac's per axis, bit for bit.
__device__ __forceinline__ void nb_frac3(float4 v, const GridParams &G, int &k0, int &k1, int &k2, float &t0,
                                         float &t1, float &t2) {
  float fc = fmaf(v.z, G.invL2, 0.5f);
  float fb = fmaf(v.y, G.invL1, 0.5f) - fc * G.tb_c;
  float fa = fmaf(v.x, G.invL0, 0.5f) - (fb * G.ta_b + fc * G.ta_c);
  float f[3] = {fa, fb, fc};
  int K[3] = {G.K0, G.K1, G.K2};
  int kk[3];
  float tt[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float g = f[a] - floorf(f[a]);
    float u = g * (float)K[a];
    float fl = floorf(u);
    int k = (int)fl;
    if (k >= K[a]) k -= K[a];
    if (k < 0) k += K[a];
    kk[a] = k;
    float t = u - fl;
    tt[a] = t >= 1.f ? 0.f : t;
  }
  k0 = kk[0];
  k1 = kk[1];
  k2 = kk[2];
  t0 = tt[0];
  t1 = tt[1];
  t2 = tt[2];
}

// The force -q grad(sum phi W) from the spline-slope sums (g0, g1, g2) of
// the three fractions: -q H^-1 (K0 g0, K1 g1, K2 g2); per axis in an
// orthorhombic cell.
__device__ __forceinline__ float3 nb_frac_force(const GridParams &G, float q, float g0, float g1, float g2) {
  float ga = -q * g0 * (float)G.K0, gb = -q * g1 * (float)G.K1, gc = -q * g2 * (float)G.K2;
  return make_float3(ga * G.invL0, gb * G.invL1 + ga * G.h10, gc * G.invL2 + ga * G.h20 + gb * G.h21);
}

// a[c] for a lane-dependent c, picked by selects: a dynamic index would
// put the array (registers of an unrolled spline) in local memory.
template <int P>
__device__ __forceinline__ float nb_pick(const float (&a)[P], int c) {
  float v = 0.f;
#pragma unroll
  for (int j = 0; j < P; ++j) v = j == c ? a[j] : v;
  return v;
}
