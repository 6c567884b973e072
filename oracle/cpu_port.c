/* OpenMP CPU port of MDIR's host path for the short-range nonbonded + PME
 * term: the timed CPU baseline that bench.py reports beside the device path
 * (TEST / BASELINE INFRASTRUCTURE; the product never loads it).
 *
 * MDIR's own CPU path is MLIR-generated code that needs LLVM/MLIR to build,
 * so this is a restatement of its algorithm in its mixed-precision roles
 * (docs/paper/07-precision.md:8-16):
 *  - a neighbor matrix from a cell list, f32 positions, each particle's row
 *    holding every partner within the widened reach, excluded pairs left out
 *    (lib/Runtime/Templates/NeighborsMatrix.mlir:1-30; docs/neighbors.md);
 *  - a row loop in f32 that computes each pair for both particles, with the
 *    energy of a row summed in f64 (MDExecToLoops; D171 fixed chunks);
 *  - PME spreading into i64 fixed point at 2^40 with atomics
 *    (lib/Conversion/MDExecToLoops/HostPMESpread.cpp:115), the grid
 *    converted to f64, and the gather in f64 (HostPMEGather.cpp:204).
 * The FFT and convolution are done by the caller (numpy's pocketfft). */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

int cpu_threads(void) { return omp_get_max_threads(); }
void cpu_set_threads(int n) { omp_set_num_threads(n); }

/* Neighbor matrix: rows of at most `width` partners. Returns the longest
 * row (a row longer than width is cut; the caller grows and retries). */
int32_t cpu_neighbor_matrix(int64_t n, const double *x, const double *box,
                            double reach, const int32_t *excl_off,
                            const int32_t *excl, int32_t width, float *xw,
                            int32_t *counts, int32_t *nbr) {
  double Rw = reach + 3e-6 * (box[0] + box[1] + box[2]);
  float R2 = (float)(Rw * Rw);
  float Lf[3] = {(float)box[0], (float)box[1], (float)box[2]};
  int nc[3];
  for (int k = 0; k < 3; ++k) {
    nc[k] = (int)floor(box[k] / Rw);
    if (nc[k] < 1) nc[k] = 1;
  }
  int64_t total = (int64_t)nc[0] * nc[1] * nc[2];
  int32_t *cell = malloc(sizeof(int32_t) * n);
  int32_t *start = calloc(total + 1, sizeof(int32_t));
  int32_t *item = malloc(sizeof(int32_t) * n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    int idx[3];
    for (int k = 0; k < 3; ++k) {
      double v = x[3 * i + k];
      float w = (float)(v - floor(v / box[k]) * box[k]);
      xw[4 * i + k] = w;
      int c = (int)floor((double)w / box[k] * nc[k]);
      idx[k] = c < 0 ? 0 : (c >= nc[k] ? nc[k] - 1 : c);
    }
    cell[i] = (idx[2] * nc[1] + idx[1]) * nc[0] + idx[0];
  }
  for (int64_t i = 0; i < n; ++i) start[cell[i] + 1]++;
  for (int64_t c = 0; c < total; ++c) start[c + 1] += start[c];
  int32_t *fill = malloc(sizeof(int32_t) * total);
  memcpy(fill, start, sizeof(int32_t) * total);
  for (int64_t i = 0; i < n; ++i) item[fill[cell[i]]++] = (int32_t)i;
  free(fill);
  int32_t longest = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(max : longest)
  for (int64_t i = 0; i < n; ++i) {
    int c0 = cell[i];
    int cx = c0 % nc[0], cy = (c0 / nc[0]) % nc[1], cz = c0 / (nc[0] * nc[1]);
    int32_t cnt = 0;
    for (int oz = -1; oz <= 1; ++oz)
      for (int oy = -1; oy <= 1; ++oy)
        for (int ox = -1; ox <= 1; ++ox) {
          int u[3] = {cx + ox, cy + oy, cz + oz}, cb[3], s[3];
          for (int k = 0; k < 3; ++k) {
            int w = ((u[k] % nc[k]) + nc[k]) % nc[k];
            s[k] = (u[k] - w) / nc[k];
            cb[k] = w;
          }
          int b = (cb[2] * nc[1] + cb[1]) * nc[0] + cb[0];
          for (int32_t t = start[b]; t < start[b + 1]; ++t) {
            int32_t j = item[t];
            if (j == i && s[0] == 0 && s[1] == 0 && s[2] == 0) continue;
            float d0 = (xw[4 * j] + s[0] * Lf[0]) - xw[4 * i];
            float d1 = (xw[4 * j + 1] + s[1] * Lf[1]) - xw[4 * i + 1];
            float d2 = (xw[4 * j + 2] + s[2] * Lf[2]) - xw[4 * i + 2];
            float r2 = d0 * d0 + d1 * d1 + d2 * d2;
            if (!(r2 <= R2)) continue;
            int ex = 0;
            if (excl_off)
              for (int32_t e = excl_off[i]; e < excl_off[i + 1]; ++e)
                if (excl[e] == j) ex = 1;
            if (ex) continue;
            if (cnt < width) nbr[i * (int64_t)width + cnt] = j | ((9 * (s[2] + 1) + 3 * (s[1] + 1) + (s[0] + 1)) << 26);
            ++cnt;
          }
        }
    counts[i] = cnt;
    if (cnt > longest) longest = cnt;
  }
  free(cell);
  free(start);
  free(item);
  return longest;
}

/* The row loop in f32: LJ from a sigma/epsilon table and Ewald direct with
 * erfcf, each pair computed for both particles (forces of row i only).
 * energy[0] += LJ, energy[1] += Coulomb (each pair counted at weight 1/2
 * in both rows). xw holds (x, y, z, -) wrapped f32 positions. */
void cpu_pairs(int64_t n, const float *xw, const float *q, const int32_t *type,
               int32_t ntypes, const float *c6, const float *c12,
               const double *box, double rc, double beta, double coulomb,
               int32_t width, const int32_t *counts, const int32_t *nbr,
               double *forces, double *energy) {
  float Lf[3] = {(float)box[0], (float)box[1], (float)box[2]};
  float rc2 = (float)(rc * rc), b = (float)beta, f = (float)coulomb;
  float tbsp = (float)(2.0 * beta / sqrt(M_PI));
  double elj = 0.0, ec = 0.0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : elj, ec)
  for (int64_t i = 0; i < n; ++i) {
    float fx = 0, fy = 0, fz = 0;
    double rl = 0, rcoul = 0;
    int32_t m = counts[i] < width ? counts[i] : width;
    for (int32_t t = 0; t < m; ++t) {
      int32_t e = nbr[i * (int64_t)width + t];
      int32_t j = e & ((1 << 26) - 1), code = e >> 26;
      int s0 = code % 3 - 1, s1 = (code / 3) % 3 - 1, s2 = code / 9 - 1;
      float dx = xw[4 * i] - (xw[4 * j] + s0 * Lf[0]);
      float dy = xw[4 * i + 1] - (xw[4 * j + 1] + s1 * Lf[1]);
      float dz = xw[4 * i + 2] - (xw[4 * j + 2] + s2 * Lf[2]);
      float r2 = dx * dx + dy * dy + dz * dz;
      if (!(r2 < rc2)) continue;
      float rinv = 1.0f / sqrtf(r2), r = r2 * rinv, rinv2 = rinv * rinv;
      int tp = type[i] * ntypes + type[j];
      float s6 = rinv2 * rinv2 * rinv2;
      float a12 = c12[tp] * s6 * s6, a6 = c6[tp] * s6;
      float fs = (12.0f * a12 - 6.0f * a6) * rinv2;
      rl += 0.5 * (double)(a12 - a6);
      float qq = f * q[i] * q[j];
      if (qq != 0.0f) {
        float er = erfcf(b * r);
        rcoul += 0.5 * (double)(qq * er * rinv);
        fs += qq * (er * rinv + tbsp * expf(-b * b * r2)) * rinv2;
      }
      fx += fs * dx;
      fy += fs * dy;
      fz += fs * dz;
    }
    forces[3 * i] += fx;
    forces[3 * i + 1] += fy;
    forces[3 * i + 2] += fz;
    elj += rl;
    ec += rcoul;
  }
  energy[0] += elj;
  energy[1] += ec;
}

static void bspline4p(int p, double t, double *w, double *dw) {
  double a[16], prev[16];
  a[0] = t;
  a[1] = 1.0 - t;
  for (int m = 3; m <= p; ++m) {
    for (int j = 0; j < m - 1; ++j) prev[j] = a[j];
    prev[m - 1] = 0.0;
    if (m == p && dw)
      for (int j = 0; j < p; ++j)
        dw[j] = (j < m - 1 ? prev[j] : 0.0) - (j > 0 ? prev[j - 1] : 0.0);
    for (int j = 0; j < m; ++j)
      a[j] = ((t + j) * prev[j] + ((double)m - t - j) * (j > 0 ? prev[j - 1] : 0.0)) / (m - 1);
  }
  for (int j = 0; j < p; ++j) w[j] = a[j];
}

/* Spreading into i64 at 2^40 with atomics, then the f64 grid. */
void cpu_pme_spread(int64_t n, const double *x, const double *q,
                    const double *box, const int64_t *K, int32_t order,
                    int64_t *fixed, double *grid) {
  int64_t total = K[0] * K[1] * K[2];
  memset(fixed, 0, sizeof(int64_t) * total);
  const double scale = 1099511627776.0; /* 2^40 */
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    int64_t k0[3];
    double w[3][16];
    for (int a = 0; a < 3; ++a) {
      double f = x[3 * i + a] / box[a];
      f -= floor(f);
      double u = f * K[a], fl = floor(u);
      if (fl >= K[a]) fl -= K[a];
      k0[a] = (int64_t)fl;
      bspline4p(order, u - floor(u), w[a], NULL);
    }
    for (int jx = 0; jx < order; ++jx) {
      int64_t gx = ((k0[0] - jx) % K[0] + K[0]) % K[0];
      for (int jy = 0; jy < order; ++jy) {
        int64_t gy = ((k0[1] - jy) % K[1] + K[1]) % K[1];
        double wxy = q[i] * w[0][jx] * w[1][jy];
        for (int jz = 0; jz < order; ++jz) {
          int64_t gz = ((k0[2] - jz) % K[2] + K[2]) % K[2];
          int64_t v = (int64_t)llrint(wxy * w[2][jz] * scale);
#pragma omp atomic
          fixed[(gx * K[1] + gy) * K[2] + gz] += v;
        }
      }
    }
  }
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < total; ++k) grid[k] = (double)fixed[k] / scale;
}

void cpu_pme_gather(int64_t n, const double *x, const double *q,
                    const double *box, const int64_t *K, int32_t order,
                    const double *phi, double *forces) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    int64_t k0[3];
    double w[3][16], dw[3][16];
    for (int a = 0; a < 3; ++a) {
      double f = x[3 * i + a] / box[a];
      f -= floor(f);
      double u = f * K[a], fl = floor(u);
      if (fl >= K[a]) fl -= K[a];
      k0[a] = (int64_t)fl;
      bspline4p(order, u - floor(u), w[a], dw[a]);
    }
    double g[3] = {0, 0, 0};
    for (int jx = 0; jx < order; ++jx) {
      int64_t gx = ((k0[0] - jx) % K[0] + K[0]) % K[0];
      for (int jy = 0; jy < order; ++jy) {
        int64_t gy = ((k0[1] - jy) % K[1] + K[1]) % K[1];
        for (int jz = 0; jz < order; ++jz) {
          int64_t gz = ((k0[2] - jz) % K[2] + K[2]) % K[2];
          double p = phi[(gx * K[1] + gy) * K[2] + gz];
          g[0] += p * dw[0][jx] * w[1][jy] * w[2][jz];
          g[1] += p * w[0][jx] * dw[1][jy] * w[2][jz];
          g[2] += p * w[0][jx] * w[1][jy] * dw[2][jz];
        }
      }
    }
    for (int a = 0; a < 3; ++a) forces[3 * i + a] -= q[i] * g[a] * K[a] / box[a];
  }
}
