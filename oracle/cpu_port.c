/* OpenMP CPU port of MDIR's host path for the short-range nonbonded + PME
 * term: the timed CPU baseline that bench.py reports beside the device path
 * (test and CPU-baseline infrastructure; the product never loads it).
 *
 * MDIR's own CPU path is MLIR-generated code that needs LLVM/MLIR to build,
 * so this is a restatement of its algorithm in its mixed-precision roles
 * (docs/paper/07-precision.md:8-16):
 *  - a neighbor matrix from linked cells of half the reach (a 5 x 5 x 5
 *    window), f32 positions, each particle's row holding every partner
 *    within the widened reach, excluded pairs left out
 *    (lib/Runtime/Templates/NeighborsMatrix.mlir:1-40; docs/neighbors.md);
 *    the matrix serves later positions while no particle has moved more
 *    than half the skin, through the whole-cell shift each particle had at
 *    the build (cpu_frames);
 *  - a row loop in f32 that computes each pair for both particles
 *    (MDExecToLoops), with erfc(beta r) as exp(-beta^2 r^2) P(1/(1 + x/2)),
 *    MDIR's fast-math approximation (D90,
 *    lib/Dialect/MDExec/Transforms/Approximate.cpp:28-40, P fitted by
 *    scripts/fit-erfc.py), the exponential shared with the force; a row's
 *    energy summed in f32 and the rows in f64;
 *  - the excluded-pair correction in f64 (TermNonbonded.cpp:1615-1671),
 *    a particle's own excluded row at a time;
 *  - PME spreading into i64 fixed point at 2^40 with atomics
 *    (lib/Conversion/MDExecToLoops/HostPMESpread.cpp:115; D70, D271), the
 *    grid converted to f64, the product with the influence function in a
 *    parallel loop over rows (D271), and the gather in f64
 *    (HostPMEGather.cpp:204).
 * The 3D FFT is MDIR's own: runtime/mdrt_fft.c over third_party/pocketfft,
 * compiled from the reference's sources into oracle/_ref/ and loaded with
 * cpu_fft_load; its line transforms are called from parallel loops over
 * the rows and the column tiles of each pass, as MDIR's compiled code does
 * (D271).  Without that library the caller does the FFT (numpy's
 * pocketfft). */
#include <dlfcn.h>
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

int cpu_threads(void) { return omp_get_max_threads(); }
void cpu_set_threads(int n) { omp_set_num_threads(n); }

/* The image of an entry: 9 (s2 + 1) + 3 (s1 + 1) + (s0 + 1), each s the
 * whole cells added to the partner, in bits 26-30 of the entry. */
#define CPU_INDEX_BITS 26

/* Neighbor matrix: rows of at most `width` partners.  Writes the f32
 * positions wrapped into the cell (xw, 4 floats a particle) and the whole
 * cells each particle was moved by (shift, 3 ints a particle).  Returns the
 * longest row (a row longer than width is cut; the caller grows and
 * retries). */
int32_t cpu_neighbor_matrix(int64_t n, const double *x, const double *box, double reach,
                            const int32_t *excl_off, const int32_t *excl, int32_t width, float *xw,
                            int32_t *shift, int32_t *counts, int32_t *nbr) {
  double Rw = reach + 3e-6 * (box[0] + box[1] + box[2]);
  float R2 = (float)(Rw * Rw);
  float Lf[3] = {(float)box[0], (float)box[1], (float)box[2]};
  /* cells of half the reach and a 5-cell window, or of the reach and a
   * 3-cell window when an edge holds fewer than 5 half-reach cells (the
   * images of a window cell are then still shifted by -1, 0 or 1 cells) */
  int half = 1, nc[3];
  for (int k = 0; k < 3; ++k)
    if ((int)floor(box[k] / (0.5 * Rw * 1.0001)) < 5) half = 0;
  int span = half ? 2 : 1;
  for (int k = 0; k < 3; ++k) {
    nc[k] = (int)floor(box[k] / ((half ? 0.5 : 1.0) * Rw * 1.0001));
    if (nc[k] < 1) nc[k] = 1;
  }
  int64_t total = (int64_t)nc[0] * nc[1] * nc[2];
  int32_t *cell = malloc(sizeof(int32_t) * n);
  int32_t *start = calloc(total + 1, sizeof(int32_t));
  int32_t *item = malloc(sizeof(int32_t) * n);
  float *cx4 = malloc(sizeof(float) * 4 * n); /* positions in cell order */
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    int idx[3];
    for (int k = 0; k < 3; ++k) {
      double v = x[3 * i + k];
      double s = floor(v / box[k]);
      float w = (float)(v - s * box[k]);
      if (w >= Lf[k]) { /* v just below a multiple of the edge */
        s += 1.0;
        w = (float)(v - s * box[k]);
      }
      xw[4 * i + k] = w;
      shift[3 * i + k] = (int32_t)s;
      int c = (int)floor((double)w / box[k] * nc[k]);
      idx[k] = c < 0 ? 0 : (c >= nc[k] ? nc[k] - 1 : c);
    }
    xw[4 * i + 3] = 0.0f;
    cell[i] = (idx[2] * nc[1] + idx[1]) * nc[0] + idx[0];
  }
  for (int64_t i = 0; i < n; ++i) start[cell[i] + 1]++;
  for (int64_t c = 0; c < total; ++c) start[c + 1] += start[c];
  int32_t *fill = malloc(sizeof(int32_t) * total);
  memcpy(fill, start, sizeof(int32_t) * total);
  for (int64_t i = 0; i < n; ++i) item[fill[cell[i]]++] = (int32_t)i;
  free(fill);
#pragma omp parallel for schedule(static)
  for (int64_t t = 0; t < n; ++t)
    for (int k = 0; k < 4; ++k) cx4[4 * t + k] = xw[4 * item[t] + k];
  int32_t longest = 0;
#pragma omp parallel reduction(max : longest)
  {
    float *r2s = malloc(sizeof(float) * (n < 65536 ? n : 65536));
#pragma omp for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; ++i) {
      int c0 = cell[i];
      int ci = c0 % nc[0], cj = (c0 / nc[0]) % nc[1], ck = c0 / (nc[0] * nc[1]);
      float xi = xw[4 * i], yi = xw[4 * i + 1], zi = xw[4 * i + 2];
      int32_t cnt = 0;
      for (int oz = -span; oz <= span; ++oz)
        for (int oy = -span; oy <= span; ++oy)
          for (int ox = -span; ox <= span; ++ox) {
            int u[3] = {ci + ox, cj + oy, ck + oz}, cb[3], s[3];
            for (int k = 0; k < 3; ++k) {
              int w = ((u[k] % nc[k]) + nc[k]) % nc[k];
              s[k] = (u[k] - w) / nc[k];
              cb[k] = w;
            }
            int b = (cb[2] * nc[1] + cb[1]) * nc[0] + cb[0];
            float sx = s[0] * Lf[0], sy = s[1] * Lf[1], sz = s[2] * Lf[2];
            int32_t t0 = start[b], t1 = start[b + 1];
            for (int32_t c = t0; c < t1; c += 65536) {
              int32_t m = t1 - c < 65536 ? t1 - c : 65536;
              const float *p = cx4 + 4 * (int64_t)c;
#pragma omp simd
              for (int32_t k = 0; k < m; ++k) {
                float d0 = (p[4 * k] + sx) - xi, d1 = (p[4 * k + 1] + sy) - yi, d2 = (p[4 * k + 2] + sz) - zi;
                r2s[k] = d0 * d0 + d1 * d1 + d2 * d2;
              }
              for (int32_t k = 0; k < m; ++k) {
                if (!(r2s[k] <= R2)) continue;
                int32_t j = item[c + k];
                if (j == i && s[0] == 0 && s[1] == 0 && s[2] == 0) continue;
                int ex = 0;
                if (excl_off)
                  for (int32_t e = excl_off[i]; e < excl_off[i + 1]; ++e)
                    if (excl[e] == j) ex = 1;
                if (ex) continue;
                if (cnt < width)
                  nbr[i * (int64_t)width + cnt] =
                      j | ((9 * (s[2] + 1) + 3 * (s[1] + 1) + (s[0] + 1)) << CPU_INDEX_BITS);
                ++cnt;
              }
            }
          }
      counts[i] = cnt;
      if (cnt > longest) longest = cnt;
    }
    free(r2s);
  }
  free(cell);
  free(start);
  free(item);
  free(cx4);
  return longest;
}

/* The f32 positions of x in the frame of the last build: x minus the whole
 * cells each particle was moved by then, so that the images of the matrix
 * stay right while no particle has moved more than half the skin. */
void cpu_frames(int64_t n, const double *x, const double *box, const int32_t *shift, float *xw) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) xw[4 * i + k] = (float)(x[3 * i + k] - shift[3 * i + k] * box[k]);
}

/* erfc(x) exp(x^2) ~ P(1 / (1 + x/2)), P of degree 9 from its constant
 * term up: MDIR's fast-math approximation of an f32 erfc (D90; relative
 * error below 3.3e-7 on [0, 6]). */
static const float ERFC_P[10] = {
    -5.844017783662725e-05f, 0.28321992286605291f,  0.27292130542277271f, 0.28757948962599933f,
    0.072615343657635112f,   0.21878733123987557f,  -0.021014074929707336f, -0.25983392190712945f,
    0.18656882080781992f,    -0.04078578921930151f};

/* The row loop in f32: LJ from c6/c12 tables and Ewald direct, each pair
 * computed for both particles (forces of row i only).  energy[0] += LJ,
 * energy[1] += Coulomb (each pair at weight 1/2 in both rows).  xw holds
 * (x, y, z, -) f32 positions in the frame of the build. */
void cpu_pairs(int64_t n, const float *xw, const float *q, const int32_t *type, int32_t ntypes,
               const float *c6, const float *c12, const double *box, double rc, double beta,
               double coulomb, int32_t width, const int32_t *counts, const int32_t *nbr,
               double *forces, double *energy) {
  float img[27][3];
  for (int c = 0; c < 27; ++c) {
    img[c][0] = (c % 3 - 1) * (float)box[0];
    img[c][1] = ((c / 3) % 3 - 1) * (float)box[1];
    img[c][2] = (c / 9 - 1) * (float)box[2];
  }
  const float rc2 = (float)(rc * rc), b = (float)beta, b2 = (float)(beta * beta), f = (float)coulomb;
  const float tbsp = (float)(2.0 * beta / sqrt(M_PI));
  const int32_t low = (1 << CPU_INDEX_BITS) - 1;
  double elj = 0.0, ec = 0.0;
#pragma omp parallel for schedule(dynamic, 32) reduction(+ : elj, ec)
  for (int64_t i = 0; i < n; ++i) {
    const float xi = xw[4 * i], yi = xw[4 * i + 1], zi = xw[4 * i + 2];
    const float qi = f * q[i];
    const int32_t ti = type[i] * ntypes;
    float fx = 0, fy = 0, fz = 0, rl = 0, rq = 0;
    const int32_t m = counts[i] < width ? counts[i] : width;
    const int32_t *row = nbr + i * (int64_t)width;
#pragma omp simd reduction(+ : fx, fy, fz, rl, rq)
    for (int32_t t = 0; t < m; ++t) {
      const int32_t e = row[t];
      const int32_t j = e & low, c = (int32_t)((uint32_t)e >> CPU_INDEX_BITS);
      const float dx = xi - (xw[4 * j] + img[c][0]);
      const float dy = yi - (xw[4 * j + 1] + img[c][1]);
      const float dz = zi - (xw[4 * j + 2] + img[c][2]);
      const float r2 = dx * dx + dy * dy + dz * dz;
      const int in = r2 < rc2;
      const float rr = in ? r2 : 1.0f;
      const float rinv = 1.0f / sqrtf(rr), rinv2 = rinv * rinv;
      const float s6 = rinv2 * rinv2 * rinv2;
      const int tp = ti + type[j];
      const float a12 = c12[tp] * s6 * s6, a6 = c6[tp] * s6;
      const float qq = qi * q[j];
      const float xb = b * rr * rinv;
      const float ex = expf(-b2 * rr);
      const float u = 1.0f / (1.0f + 0.5f * xb);
      float p = ERFC_P[9];
      p = p * u + ERFC_P[8];
      p = p * u + ERFC_P[7];
      p = p * u + ERFC_P[6];
      p = p * u + ERFC_P[5];
      p = p * u + ERFC_P[4];
      p = p * u + ERFC_P[3];
      p = p * u + ERFC_P[2];
      p = p * u + ERFC_P[1];
      p = p * u + ERFC_P[0];
      const float er = ex * p;
      const float fs = ((12.0f * a12 - 6.0f * a6) + qq * (er * rinv + tbsp * ex)) * rinv2;
      const float w = in ? 1.0f : 0.0f;
      fx += w * fs * dx;
      fy += w * fs * dy;
      fz += w * fs * dz;
      rl += w * (a12 - a6);
      rq += w * qq * er * rinv;
    }
    forces[3 * i] += fx;
    forces[3 * i + 1] += fy;
    forces[3 * i + 2] += fz;
    elj += 0.5 * (double)rl;
    ec += 0.5 * (double)rq;
  }
  energy[0] += elj;
  energy[1] += ec;
}

/* The excluded-pair correction -f q_i q_j erf(beta r)/r in f64, each
 * particle's own excluded row (both directions), so that every thread
 * writes its own particles only.  energy[2] += the correction. */
void cpu_excluded(int64_t n, const double *x, const double *q, const double *box, const int32_t *off,
                  const int32_t *partners, double beta, double coulomb, double *forces, double *energy) {
  const double tbsp = 2.0 * beta / sqrt(M_PI);
  double e = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : e)
  for (int64_t i = 0; i < n; ++i) {
    for (int32_t k = off[i]; k < off[i + 1]; ++k) {
      int32_t j = partners[k];
      double d[3], r2 = 0.0;
      for (int a = 0; a < 3; ++a) {
        d[a] = x[3 * i + a] - x[3 * j + a];
        d[a] -= box[a] * nearbyint(d[a] / box[a]);
        r2 += d[a] * d[a];
      }
      double r = sqrt(r2), qq = coulomb * q[i] * q[j];
      double er = erf(beta * r);
      e += -0.5 * qq * er / r;
      double fs = -qq * (er / r - tbsp * exp(-beta * beta * r2)) / r2;
      for (int a = 0; a < 3; ++a) forces[3 * i + a] += fs * d[a];
    }
  }
  energy[2] += e;
}

static void bspline4p(int p, double t, double *w, double *dw) {
  double a[16], prev[16];
  a[0] = t;
  a[1] = 1.0 - t;
  for (int m = 3; m <= p; ++m) {
    for (int j = 0; j < m - 1; ++j) prev[j] = a[j];
    prev[m - 1] = 0.0;
    if (m == p && dw)
      for (int j = 0; j < p; ++j) dw[j] = (j < m - 1 ? prev[j] : 0.0) - (j > 0 ? prev[j - 1] : 0.0);
    for (int j = 0; j < m; ++j)
      a[j] = ((t + j) * prev[j] + ((double)m - t - j) * (j > 0 ? prev[j - 1] : 0.0)) / (m - 1);
  }
  for (int j = 0; j < p; ++j) w[j] = a[j];
}

/* Spreading into i64 at 2^40 with atomics, then the f64 grid. */
void cpu_pme_spread(int64_t n, const double *x, const double *q, const double *box, const int64_t *K,
                    int32_t order, int64_t *fixed, double *grid) {
  int64_t total = K[0] * K[1] * K[2];
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < total; ++k) fixed[k] = 0;
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
      int64_t gx = k0[0] - jx < 0 ? k0[0] - jx + K[0] : k0[0] - jx;
      for (int jy = 0; jy < order; ++jy) {
        int64_t gy = k0[1] - jy < 0 ? k0[1] - jy + K[1] : k0[1] - jy;
        double wxy = q[i] * w[0][jx] * w[1][jy];
        for (int jz = 0; jz < order; ++jz) {
          int64_t gz = k0[2] - jz < 0 ? k0[2] - jz + K[2] : k0[2] - jz;
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

void cpu_pme_gather(int64_t n, const double *x, const double *q, const double *box, const int64_t *K,
                    int32_t order, const double *phi, double *forces) {
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
      int64_t gx = k0[0] - jx < 0 ? k0[0] - jx + K[0] : k0[0] - jx;
      for (int jy = 0; jy < order; ++jy) {
        int64_t gy = k0[1] - jy < 0 ? k0[1] - jy + K[1] : k0[1] - jy;
        for (int jz = 0; jz < order; ++jz) {
          int64_t gz = k0[2] - jz < 0 ? k0[2] - jz + K[2] : k0[2] - jz;
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

/* ---- MDIR's host FFT (runtime/mdrt_fft.c), loaded from oracle/_ref ---- */

/* The descriptor of a one-dimensional buffer as MLIR's C interface passes
 * it (the layout mdrt_fft.c's functions take). */
typedef struct {
  double *allocated, *aligned;
  int64_t offset, sizes[1], strides[1];
} cpu_memref_f64;

static void (*fft_prepare)(int64_t, int64_t, int64_t);
static int64_t (*fft_column_blocks)(int64_t, int64_t);
static void (*fft_rows_forward)(cpu_memref_f64 *, cpu_memref_f64 *, int64_t, int64_t, int64_t);
static void (*fft_rows_backward)(cpu_memref_f64 *, cpu_memref_f64 *, int64_t, int64_t, int64_t);
static void (*fft_columns)(cpu_memref_f64 *, int64_t, int64_t, int64_t, int64_t, int64_t, int64_t, int64_t);

/* Loads the FFT functions from the shared library at `path`; 0 when every
 * one was found. */
int32_t cpu_fft_load(const char *path) {
  void *h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
  if (!h) return 1;
  fft_prepare = (void (*)(int64_t, int64_t, int64_t))dlsym(h, "mdrtFFTPrepare");
  fft_column_blocks = (int64_t(*)(int64_t, int64_t))dlsym(h, "mdrtFFTColumnBlocks");
  fft_rows_forward = (void (*)(cpu_memref_f64 *, cpu_memref_f64 *, int64_t, int64_t, int64_t))dlsym(
      h, "_mlir_ciface_mdrtFFT64RowsForward");
  fft_rows_backward = (void (*)(cpu_memref_f64 *, cpu_memref_f64 *, int64_t, int64_t, int64_t))dlsym(
      h, "_mlir_ciface_mdrtFFT64RowsBackward");
  fft_columns = (void (*)(cpu_memref_f64 *, int64_t, int64_t, int64_t, int64_t, int64_t, int64_t,
                          int64_t))dlsym(h, "_mlir_ciface_mdrtFFT64Columns");
  return !(fft_prepare && fft_column_blocks && fft_rows_forward && fft_rows_backward && fft_columns);
}

static cpu_memref_f64 memref(double *p, int64_t size) {
  cpu_memref_f64 m = {p, p, 0, {size}, {1}};
  return m;
}

/* The reciprocal sum on the f64 grid Q (k1 k2 k3), overwritten with the
 * potential grid phi: the forward transform, the product with B C (bc,
 * k1 k2 (k3/2 + 1)), and the backward transform, not normalized; spec is
 * the half-complex scratch (2 k1 k2 (k3/2 + 1) doubles), rowsum k1 k2.  Each
 * pass is a parallel loop over blocks of lines, as MDIR's compiled code
 * calls mdrt_fft.c (D271).  Returns the reciprocal energy
 * 1/2 sum B C |S|^2 (each half-complex point weighted by its mirror),
 * summed along a row and over rows in a fixed order. */
double cpu_pme_reciprocal(const int64_t *K, double *Q, double *spec, const double *bc, double *rowsum) {
  const int64_t k1 = K[0], k2 = K[1], k3 = K[2], h = k3 / 2 + 1;
  cpu_memref_f64 real = memref(Q, k1 * k2 * k3), cplx = memref(spec, 2 * k1 * k2 * h);
  fft_prepare(k1, k2, k3);
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < k1 * k2; ++r) fft_rows_forward(&real, &cplx, k3, r, r + 1);
  int64_t ny = fft_column_blocks(k1, k3), nx = fft_column_blocks(k2, k3);
#pragma omp parallel for schedule(static)
  for (int64_t u = 0; u < ny; ++u) fft_columns(&cplx, k1, k2, k3, 1, 1, u, u + 1);
#pragma omp parallel for schedule(static)
  for (int64_t u = 0; u < nx; ++u) fft_columns(&cplx, k1, k2, k3, 0, 1, u, u + 1);
  /* the product with B C and the energy of each row */
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < k1 * k2; ++r) {
    double s = 0.0;
    for (int64_t z = 0; z < h; ++z) {
      double *c = spec + 2 * (r * h + z);
      double w = (z == 0 || (k3 % 2 == 0 && z == h - 1)) ? 1.0 : 2.0;
      double g = bc[r * h + z];
      s += w * g * (c[0] * c[0] + c[1] * c[1]);
      c[0] *= g;
      c[1] *= g;
    }
    rowsum[r] = s;
  }
  double e = 0.0;
  for (int64_t r = 0; r < k1 * k2; ++r) e += rowsum[r];
#pragma omp parallel for schedule(static)
  for (int64_t u = 0; u < ny; ++u) fft_columns(&cplx, k1, k2, k3, 1, 0, u, u + 1);
#pragma omp parallel for schedule(static)
  for (int64_t u = 0; u < nx; ++u) fft_columns(&cplx, k1, k2, k3, 0, 0, u, u + 1);
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < k1 * k2; ++r) fft_rows_backward(&cplx, &real, k3, r, r + 1);
  return 0.5 * e;
}
