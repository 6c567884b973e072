/* CPU oracle for the short-range nonbonded + PME path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this file: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg use it, and only as the checker.
 *
 * It restates, in plain C (FP64 unless a function says f32), the algorithms
 * of MDIR (vv137/mdir) that the device path replaces:
 *
 *  - the pair set of a neighbor build: every image of every pair whose f32
 *    distance, with the reach widened by 3e-6 of the sum of the edges, is
 *    within that reach (docs/neighbor-groups.md, Sections 4, 5.2 and 7.2;
 *    lib/Conversion/MDExecKernels/GroupsBuild.cpp:2592-2607 for the widening);
 *  - the Lennard-Jones + Ewald direct pair term, the excluded-pair
 *    correction and their virial (lib/Driver/TermNonbonded.cpp:378-466 and
 *    1615-1671; lib/Driver/TermLennardJones.cpp:26-80, the r^2 cubic switch
 *    of [Brooks1983] at TermLennardJones.cpp:57-75);
 *  - smooth PME charge spreading and force / potential gathering with
 *    cardinal B-splines of any order (docs/pme.md, Section 1;
 *    lib/Conversion/MDExecToLoops/HostPMESpread.cpp:33-190 and
 *    HostPMEGather.cpp:204-306).  The FFT and the influence function are in
 *    oracle.py (numpy), which calls these.
 *
 * Compile with -ffp-contract=off: the f32 distance test must round exactly
 * as written (no fused multiply-add), since the device build rounds the
 * same way and pair sets are compared bit for bit.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------
 * Positions of test/Runtime/neighbors-groups-gpu.mlir:47-80: a linear
 * congruential generator (a = 1103515245, c = 12345, m = 2^31, seed 42),
 * each coordinate moved by (i + 3k) mod 7 - 3 edges of the cube.
 * ---------------------------------------------------------------------- */
void orc_lcg_positions(int64_t n, double length, double *x) {
  uint64_t s = 42;
  for (int64_t i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) {
      s = (s * 1103515245ull + 12345ull) % 2147483648ull;
      double f = (double)s / 2147483648.0;
      double boxes = (double)((i + 3 * k) % 7) - 3.0;
      x[3 * i + k] = f * length + boxes * length;
    }
}

/* ------------------------------------------------------------------------
 * The canonical f32 pair test.
 *
 * wrapped:  xw = (float)(x + S L) with S = -floor(x / L), the sum in f64
 * image s:  d = ((xw_j + (float)s * Lf) - xw_i) per axis, Lf = (float)L
 * length:   r2 = (dx*dx + dy*dy) + dz*dz in f32, no fused multiply-add
 * test:     r2 <= R2f,  R2f = (float)(R' * R'),  R' = R + 3e-6 (Lx+Ly+Lz)
 * ---------------------------------------------------------------------- */
static int finite3(const double *p) {
  return isfinite(p[0]) && isfinite(p[1]) && isfinite(p[2]);
}

void orc_wrap_f32(int64_t n, const double *x, const double *box, float *xw,
                  int32_t *valid) {
  for (int64_t i = 0; i < n; ++i) {
    int ok = finite3(x + 3 * i);
    for (int k = 0; k < 3; ++k) {
      double L = box[k];
      double v = x[3 * i + k];
      double S = ok ? -floor(v / L) : 0.0;
      if (fabs(S) > 511.0) ok = 0;
      xw[3 * i + k] = ok ? (float)(v + S * L) : 0.0f;
    }
    valid[i] = ok;
  }
}

double orc_widened_reach(double reach, const double *box) {
  return reach + 3e-6 * (box[0] + box[1] + box[2]);
}

static inline float f32_dist2(const float *xi, const float *xj, const float *Lf,
                              const int *s) {
  volatile float d[3];
  for (int k = 0; k < 3; ++k) {
    volatile float shifted = xj[k] + (float)s[k] * Lf[k];
    d[k] = shifted - xi[k];
  }
  volatile float a = d[0] * d[0];
  volatile float b = d[1] * d[1];
  volatile float c = d[2] * d[2];
  volatile float ab = a + b;
  return ab + c;
}

/* A cell list over wrapped positions, cells of at least `width` a side. */
struct Cells {
  int nc[3];
  int32_t *start; /* nc0*nc1*nc2 + 1 */
  int32_t *item;
};

static void cells_build(struct Cells *c, int64_t n, const double *pos3,
                        const int32_t *valid, const double *box, double width) {
  for (int k = 0; k < 3; ++k) {
    int m = (int)floor(box[k] / width);
    c->nc[k] = m < 1 ? 1 : m;
  }
  int64_t total = (int64_t)c->nc[0] * c->nc[1] * c->nc[2];
  c->start = (int32_t *)calloc((size_t)total + 1, sizeof(int32_t));
  c->item = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  int32_t *cell = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  for (int64_t i = 0; i < n; ++i) {
    if (!valid[i]) {
      cell[i] = -1;
      continue;
    }
    int idx[3];
    for (int k = 0; k < 3; ++k) {
      int v = (int)floor(pos3[3 * i + k] / box[k] * c->nc[k]);
      if (v < 0) v = 0;
      if (v >= c->nc[k]) v = c->nc[k] - 1;
      idx[k] = v;
    }
    cell[i] = (idx[2] * c->nc[1] + idx[1]) * c->nc[0] + idx[0];
    c->start[cell[i] + 1]++;
  }
  for (int64_t k = 0; k < total; ++k) c->start[k + 1] += c->start[k];
  int32_t *fill = (int32_t *)malloc(sizeof(int32_t) * (size_t)total);
  for (int64_t k = 0; k < total; ++k) fill[k] = c->start[k];
  for (int64_t i = 0; i < n; ++i)
    if (cell[i] >= 0) c->item[fill[cell[i]]++] = (int32_t)i;
  free(fill);
  free(cell);
}

static void cells_free(struct Cells *c) {
  free(c->start);
  free(c->item);
}

static int excluded_pair(const int32_t *off, const int32_t *ex, int32_t i,
                         int32_t j) {
  if (!off) return 0;
  for (int32_t k = off[i]; k < off[i + 1]; ++k)
    if (ex[k] == j) return 1;
  return 0;
}

/* The pair set: every unordered pair {i, j} (i < j), not excluded, both
 * positions finite, and every image s in {-1,0,1}^3 of j relative to i with
 * the canonical f32 distance within the widened reach.  Writes at most `cap`
 * triples (i, j, code), code = 9(sz+1) + 3(sy+1) + (sx+1), and returns the
 * count.  The reach must be below the least edge (then no image beyond one
 * cell away can be within it). */
int64_t orc_pairset(int64_t n, const double *x, const double *box, double reach,
                    const int32_t *excl_off, const int32_t *excl, int64_t cap,
                    int32_t *out) {
  float *xw = (float *)malloc(sizeof(float) * 3 * (size_t)(n > 0 ? n : 1));
  double *xd = (double *)malloc(sizeof(double) * 3 * (size_t)(n > 0 ? n : 1));
  int32_t *valid = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  orc_wrap_f32(n, x, box, xw, valid);
  for (int64_t i = 0; i < 3 * n; ++i) xd[i] = xw[i];
  double Rw = orc_widened_reach(reach, box);
  float R2f = (float)(Rw * Rw);
  float Lf[3] = {(float)box[0], (float)box[1], (float)box[2]};
  struct Cells c;
  cells_build(&c, n, xd, valid, box, Rw);
  int64_t count = 0;
  for (int cz = 0; cz < c.nc[2]; ++cz)
    for (int cy = 0; cy < c.nc[1]; ++cy)
      for (int cx = 0; cx < c.nc[0]; ++cx) {
        int ca = (cz * c.nc[1] + cy) * c.nc[0] + cx;
        for (int oz = -1; oz <= 1; ++oz)
          for (int oy = -1; oy <= 1; ++oy)
            for (int ox = -1; ox <= 1; ++ox) {
              int u[3] = {cx + ox, cy + oy, cz + oz};
              int cb[3], s[3];
              for (int k = 0; k < 3; ++k) {
                int m = c.nc[k];
                int w = ((u[k] % m) + m) % m;
                s[k] = (u[k] - w) / m;
                cb[k] = w;
              }
              int b = (cb[2] * c.nc[1] + cb[1]) * c.nc[0] + cb[0];
              for (int32_t a = c.start[ca]; a < c.start[ca + 1]; ++a) {
                int32_t i = c.item[a];
                for (int32_t bb = c.start[b]; bb < c.start[b + 1]; ++bb) {
                  int32_t j = c.item[bb];
                  if (j <= i) continue;
                  float r2 = f32_dist2(xw + 3 * i, xw + 3 * j, Lf, s);
                  if (!(r2 <= R2f)) continue;
                  if (excluded_pair(excl_off, excl, i, j)) continue;
                  if (count < cap && out) {
                    out[3 * count] = i;
                    out[3 * count + 1] = j;
                    out[3 * count + 2] = 9 * (s[2] + 1) + 3 * (s[1] + 1) + (s[0] + 1);
                  }
                  ++count;
                }
              }
            }
      }
  cells_free(&c);
  free(xw);
  free(xd);
  free(valid);
  return count;
}

/* ------------------------------------------------------------------------
 * FP64 short-range nonbonded: Lennard-Jones from a table of sigma/epsilon
 * by type pair, 4 eps ((s/r)^12 - (s/r)^6), optionally times the cubic
 * switch in r^2, S = (1 - y)^2 (1 + 2y), y = (r^2 - rs^2)/(rc^2 - rs^2)
 * clamped to [0, 1] (TermLennardJones.cpp:57-75); Ewald direct
 * f q_i q_j (erfc(beta r)/r - shift) for r < rc (TermNonbonded.cpp:378-466);
 * every image within rc is taken.
 *
 * energies[0] = LJ, energies[1] = Coulomb direct.  virial[9] = sum d (x) F
 * with d = x_i - x_j (image) and F the force on i.  forces[3n] += forces.
 * lj_switch: 0 = none, 1 = r^2 cubic switch from rs (MDIR's
 * SQUARED_DISTANCE_SWITCH modifier), 2 = the potential switch of MDIR's md
 * dialect, S = 1 - 10 t^3 + 15 t^4 - 6 t^5, t = (r - rs)/(rc - rs), S = 1
 * for r <= rs (lib/Dialect/MD/Transforms/ExpandTruncation.cpp:19-46; the
 * expression pairs of examples/argon/argon.toml).
 * ---------------------------------------------------------------------- */
void orc_nonbonded(int64_t n, const double *x, const double *q,
                   const int32_t *type, int32_t ntypes, const double *sigma,
                   const double *epsilon, const double *box, double rc,
                   double beta, double coulomb, int32_t coulomb_shift,
                   int32_t lj_switch, double rs, const int32_t *excl_off,
                   const int32_t *excl, double *forces, double *energies,
                   double *virial) {
  double *xd = (double *)malloc(sizeof(double) * 3 * (size_t)(n > 0 ? n : 1));
  int32_t *valid = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  for (int64_t i = 0; i < n; ++i) {
    valid[i] = finite3(x + 3 * i);
    for (int k = 0; k < 3; ++k) {
      double v = x[3 * i + k];
      xd[3 * i + k] = valid[i] ? v - floor(v / box[k]) * box[k] : 0.0;
    }
  }
  double rc2 = rc * rc;
  double shift = coulomb_shift ? erfc(beta * rc) / rc : 0.0;
  double twobeta_sqrtpi = 2.0 * beta / sqrt(M_PI);
  double rs2 = rs * rs, winv = lj_switch ? 1.0 / (rc2 - rs2) : 0.0;
  double elj = 0.0, ecoul = 0.0;
  double W[9] = {0};
  struct Cells c;
  cells_build(&c, n, xd, valid, box, rc);
  for (int cz = 0; cz < c.nc[2]; ++cz)
    for (int cy = 0; cy < c.nc[1]; ++cy)
      for (int cx = 0; cx < c.nc[0]; ++cx) {
        int ca = (cz * c.nc[1] + cy) * c.nc[0] + cx;
        for (int oz = -1; oz <= 1; ++oz)
          for (int oy = -1; oy <= 1; ++oy)
            for (int ox = -1; ox <= 1; ++ox) {
              int u[3] = {cx + ox, cy + oy, cz + oz};
              int cb[3], s[3];
              for (int k = 0; k < 3; ++k) {
                int m = c.nc[k];
                int w = ((u[k] % m) + m) % m;
                s[k] = (u[k] - w) / m;
                cb[k] = w;
              }
              int b = (cb[2] * c.nc[1] + cb[1]) * c.nc[0] + cb[0];
              for (int32_t a = c.start[ca]; a < c.start[ca + 1]; ++a) {
                int32_t i = c.item[a];
                for (int32_t bb = c.start[b]; bb < c.start[b + 1]; ++bb) {
                  int32_t j = c.item[bb];
                  if (j <= i) continue;
                  double d[3];
                  for (int k = 0; k < 3; ++k)
                    d[k] = xd[3 * i + k] - (xd[3 * j + k] + s[k] * box[k]);
                  double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
                  if (!(r2 < rc2)) continue;
                  if (excluded_pair(excl_off, excl, i, j)) continue;
                  double r = sqrt(r2);
                  double fscal = 0.0; /* -dU/dr / r */
                  int ti = type[i], tj = type[j];
                  double sg = sigma[ti * ntypes + tj], ep = epsilon[ti * ntypes + tj];
                  if (ep != 0.0) {
                    double sr = sg / r, s6 = pow(sr, 6.0), s12 = s6 * s6;
                    double e = 4.0 * ep * (s12 - s6);
                    double dedr = 4.0 * ep * (-12.0 * s12 + 6.0 * s6) / r;
                    if (lj_switch == 2) {
                      if (r > rs) {
                        double t = (r - rs) / (rc - rs);
                        double S = 1.0 + t * t * t * (-10.0 + t * (15.0 - 6.0 * t));
                        double dSdr = t * t * (-30.0 + t * (60.0 - 30.0 * t)) / (rc - rs);
                        dedr = dedr * S + e * dSdr;
                        e *= S;
                      }
                    } else if (lj_switch) {
                      double y = (r2 - rs2) * winv;
                      if (y < 0.0) y = 0.0;
                      if (y > 1.0) y = 1.0;
                      double S = (1.0 - y) * (1.0 - y) * (1.0 + 2.0 * y);
                      double dSdy = (y > 0.0 && y < 1.0) ? -6.0 * y * (1.0 - y) : 0.0;
                      double dSdr = dSdy * 2.0 * r * winv;
                      dedr = dedr * S + e * dSdr;
                      e *= S;
                    }
                    elj += e;
                    fscal += -dedr / r;
                  }
                  double qq = coulomb * q[i] * q[j];
                  if (qq != 0.0) {
                    double er = erfc(beta * r);
                    ecoul += qq * (er / r - shift);
                    double dedr = qq * (-er / r2 - twobeta_sqrtpi * exp(-beta * beta * r2) / r);
                    fscal += -dedr / r;
                  }
                  for (int k = 0; k < 3; ++k) {
                    forces[3 * i + k] += fscal * d[k];
                    forces[3 * j + k] -= fscal * d[k];
                  }
                  for (int a2 = 0; a2 < 3; ++a2)
                    for (int b2 = 0; b2 < 3; ++b2) W[3 * a2 + b2] += d[a2] * fscal * d[b2];
                }
              }
            }
      }
  cells_free(&c);
  energies[0] += elj;
  energies[1] += ecoul;
  for (int k = 0; k < 9; ++k) virial[k] += W[k];
  free(xd);
  free(valid);
}

/* The excluded-pair correction -f q_i q_j erf(beta r)/r over the pairs
 * (pairs[2k], pairs[2k+1]) in the minimum image (TermNonbonded.cpp:1615-1671).
 * energies[0] += it; forces and virial as orc_nonbonded. */
void orc_excluded(int64_t npairs, const int32_t *pairs, const double *x,
                  const double *q, const double *box, double beta,
                  double coulomb, double *forces, double *energies,
                  double *virial) {
  double e = 0.0;
  double twobeta_sqrtpi = 2.0 * beta / sqrt(M_PI);
  for (int64_t p = 0; p < npairs; ++p) {
    int32_t i = pairs[2 * p], j = pairs[2 * p + 1];
    double d[3];
    for (int k = 0; k < 3; ++k) {
      double v = x[3 * i + k] - x[3 * j + k];
      d[k] = v - box[k] * nearbyint(v / box[k]);
    }
    double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    double r = sqrt(r2);
    double qq = coulomb * q[i] * q[j];
    if (qq == 0.0 || r == 0.0) continue;
    double ef = erf(beta * r);
    e += -qq * ef / r;
    /* U = -qq erf(br)/r; dU/dr = -qq (2b/sqrtpi e^{-b^2r^2}/r - erf/r^2) */
    double dedr = -qq * (twobeta_sqrtpi * exp(-beta * beta * r2) / r - ef / r2);
    double fscal = -dedr / r;
    for (int k = 0; k < 3; ++k) {
      forces[3 * i + k] += fscal * d[k];
      forces[3 * j + k] -= fscal * d[k];
    }
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) virial[3 * a + b] += d[a] * fscal * d[b];
  }
  energies[0] += e;
}

/* ------------------------------------------------------------------------
 * Cardinal B-splines.  For t in [0, 1): w[j] = M_p(t + j), dw[j] its slope,
 * j = 0 .. p-1, by M_n(x) = (x M_{n-1}(x) + (n - x) M_{n-1}(x - 1))/(n - 1).
 * The weight w[j] belongs to the grid point floor(u) - j.
 * ---------------------------------------------------------------------- */
static void bspline(int p, double t, double *w, double *dw) {
  double a[16], prev[16];
  a[0] = t;
  a[1] = 1.0 - t;
  for (int m = 3; m <= p; ++m) {
    for (int j = 0; j < m - 1; ++j) prev[j] = a[j];
    prev[m - 1] = 0.0;
    if (m == p && dw) {
      for (int j = 0; j < p; ++j)
        dw[j] = (j < m - 1 ? prev[j] : 0.0) - (j > 0 ? prev[j - 1] : 0.0);
    }
    for (int j = 0; j < m; ++j) {
      double left = prev[j];
      double right = j > 0 ? prev[j - 1] : 0.0;
      a[j] = ((t + j) * left + ((double)m - t - j) * right) / (double)(m - 1);
    }
  }
  if (p == 2 && dw) {
    dw[0] = 1.0;
    dw[1] = -1.0;
  }
  for (int j = 0; j < p; ++j) w[j] = a[j];
}

static void frac_coord(double x, double L, int64_t K, int64_t *k0, double *t) {
  double f = x / L;
  f -= floor(f);
  double u = f * (double)K;
  double fl = floor(u);
  if (fl >= (double)K) fl -= (double)K;
  *k0 = (int64_t)fl;
  *t = u - floor(u);
}

/* Q(k) += q_i prod_a M_p(u_a - k_a) into grid[K0][K1][K2] (row major, z
 * fastest).  Skips nonfinite positions. */
void orc_pme_spread(int64_t n, const double *x, const double *q,
                    const double *box, const int64_t *K, int32_t order,
                    double *grid) {
  for (int64_t i = 0; i < n; ++i) {
    if (!finite3(x + 3 * i) || q[i] == 0.0) continue;
    int64_t k0[3];
    double w[3][16];
    for (int a = 0; a < 3; ++a) {
      double t;
      frac_coord(x[3 * i + a], box[a], K[a], &k0[a], &t);
      bspline(order, t, w[a], NULL);
    }
    for (int jx = 0; jx < order; ++jx) {
      int64_t gx = ((k0[0] - jx) % K[0] + K[0]) % K[0];
      for (int jy = 0; jy < order; ++jy) {
        int64_t gy = ((k0[1] - jy) % K[1] + K[1]) % K[1];
        double wxy = q[i] * w[0][jx] * w[1][jy];
        for (int jz = 0; jz < order; ++jz) {
          int64_t gz = ((k0[2] - jz) % K[2] + K[2]) % K[2];
          grid[(gx * K[1] + gy) * K[2] + gz] += wxy * w[2][jz];
        }
      }
    }
  }
}

/* Given phi(k) = dE_rec/dQ(k): forces[i] -= q_i sum_k phi(k) grad(MMM) and
 * potential[i] = sum_k phi(k) MMM (= dE_rec/dq_i). */
void orc_pme_gather(int64_t n, const double *x, const double *q,
                    const double *box, const int64_t *K, int32_t order,
                    const double *phi, double *forces, double *potential) {
  for (int64_t i = 0; i < n; ++i) {
    if (!finite3(x + 3 * i)) continue;
    int64_t k0[3];
    double w[3][16], dw[3][16];
    for (int a = 0; a < 3; ++a) {
      double t;
      frac_coord(x[3 * i + a], box[a], K[a], &k0[a], &t);
      bspline(order, t, w[a], dw[a]);
    }
    double g[3] = {0, 0, 0}, pot = 0.0;
    for (int jx = 0; jx < order; ++jx) {
      int64_t gx = ((k0[0] - jx) % K[0] + K[0]) % K[0];
      for (int jy = 0; jy < order; ++jy) {
        int64_t gy = ((k0[1] - jy) % K[1] + K[1]) % K[1];
        for (int jz = 0; jz < order; ++jz) {
          int64_t gz = ((k0[2] - jz) % K[2] + K[2]) % K[2];
          double p = phi[(gx * K[1] + gy) * K[2] + gz];
          pot += p * w[0][jx] * w[1][jy] * w[2][jz];
          g[0] += p * dw[0][jx] * w[1][jy] * w[2][jz];
          g[1] += p * w[0][jx] * dw[1][jy] * w[2][jz];
          g[2] += p * w[0][jx] * w[1][jy] * dw[2][jz];
        }
      }
    }
    for (int a = 0; a < 3; ++a)
      forces[3 * i + a] -= q[i] * g[a] * (double)K[a] / box[a];
    if (potential) potential[i] = pot;
  }
}

/* |b(m)|^2 of the SPME B-spline moduli along one edge (Essmann 1995):
 * 1 / |sum_{k=0}^{p-2} M_p(k+1) exp(2 pi i m k / K)|^2. */
void orc_bspline_moduli(int64_t K, int32_t order, double *out) {
  double w[16];
  bspline(order, 0.0, w, NULL); /* w[j] = M_p(j) */
  for (int64_t m = 0; m < K; ++m) {
    double re = 0.0, im = 0.0;
    for (int k = 0; k <= order - 2; ++k) {
      double arg = 2.0 * M_PI * (double)m * (double)k / (double)K;
      re += w[k + 1] * cos(arg);
      im += w[k + 1] * sin(arg);
    }
    double s = re * re + im * im;
    if (s < 1e-7) {
      /* Interpolate the zero of odd orders at the Nyquist point. */
      s = -1.0;
    }
    out[m] = s > 0.0 ? 1.0 / s : 0.0;
  }
  for (int64_t m = 0; m < K; ++m)
    if (out[m] == 0.0) {
      double l = out[(m + K - 1) % K], r = out[(m + 1) % K];
      out[m] = 0.5 * (l + r);
    }
}

/* ------------------------------------------------------------------------
 * Triclinic cells (docs/neighbor-groups.md, Section 5.1; docs/triclinic.md):
 * the cell H of rows a = (ax, 0, 0), b = (bx, by, 0), c = (cx, cy, cz),
 * given as the six numbers (ax, by, cz, bx, cx, cy) of MDIR's
 * vector<6xf64>; a lattice vector n = (na, nb, nc) is n H.
 * ---------------------------------------------------------------------- */

/* The positions of test/Runtime/neighbors-groups-triclinic-gpu.mlir:47-100:
 * fractional coordinates from the generator of orc_lcg_positions, each
 * moved by (i + 3k) mod 7 - 3 lattice vectors, then x = s H. */
void orc_lcg_positions_triclinic(int64_t n, const double *cell, double *x) {
  uint64_t s = 42;
  double ax = cell[0], by = cell[1], cz = cell[2], bx = cell[3], cx = cell[4], cy = cell[5];
  for (int64_t i = 0; i < n; ++i) {
    double f[3];
    for (int k = 0; k < 3; ++k) {
      s = (s * 1103515245ull + 12345ull) % 2147483648ull;
      f[k] = (double)s / 2147483648.0 + ((double)((i + 3 * k) % 7) - 3.0);
    }
    x[3 * i] = f[0] * ax + f[1] * bx + f[2] * cx;
    x[3 * i + 1] = f[1] * by + f[2] * cy;
    x[3 * i + 2] = f[2] * cz;
  }
}

/* The widened reach of a triclinic build: 3e-6 of the sum of the diagonal
 * and the magnitudes of the three tilts (docs/neighbor-groups.md, 5.1). */
double orc_widened_reach_triclinic(double reach, const double *cell) {
  return reach + 3e-6 * (cell[0] + cell[1] + cell[2] + fabs(cell[3]) + fabs(cell[4]) + fabs(cell[5]));
}

/* Every image of every pair i < j within `reach` in f64: the displacement
 * reduced once along c, b and a, then the lattice vectors up to `span`
 * from that image along each of a, b, c.  Pairs with a position that is not
 * finite and excluded pairs have none.  Writes at most `cap` rows
 * (i, j, na, nb, nc) of the lattice vector of j's image relative to i (raw
 * positions), returns the count; *several counts the pairs with more than
 * one image within the reach. */
int64_t orc_pairset_triclinic(int64_t n, const double *x, const double *cell, double reach,
                              const int32_t *excl_off, const int32_t *excl, int32_t span, int64_t cap,
                              int32_t *out, int64_t *several) {
  double ax = cell[0], by = cell[1], cz = cell[2], bx = cell[3], cx = cell[4], cy = cell[5];
  double R2 = reach * reach;
  int64_t count = 0, multi = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (!finite3(x + 3 * i)) continue;
    for (int64_t j = i + 1; j < n; ++j) {
      if (!finite3(x + 3 * j)) continue;
      if (excluded_pair(excl_off, excl, (int32_t)i, (int32_t)j)) continue;
      double d[3] = {x[3 * j] - x[3 * i], x[3 * j + 1] - x[3 * i + 1], x[3 * j + 2] - x[3 * i + 2]};
      /* one pass along c, b, a: the lattice vector m of the reduced image */
      double mc = -rint(d[2] / cz);
      d[0] += mc * cx; d[1] += mc * cy; d[2] += mc * cz;
      double mb = -rint(d[1] / by);
      d[0] += mb * bx; d[1] += mb * by;
      double ma = -rint(d[0] / ax);
      d[0] += ma * ax;
      int found = 0;
      for (int tc = -span; tc <= span; ++tc)
        for (int tb = -span; tb <= span; ++tb)
          for (int ta = -span; ta <= span; ++ta) {
            double ex = d[0] + ta * ax + tb * bx + tc * cx;
            double ey = d[1] + tb * by + tc * cy;
            double ez = d[2] + tc * cz;
            if (!(ex * ex + ey * ey + ez * ez <= R2)) continue;
            if (count < cap && out) {
              out[5 * count] = (int32_t)i;
              out[5 * count + 1] = (int32_t)j;
              out[5 * count + 2] = (int32_t)ma + ta;
              out[5 * count + 3] = (int32_t)mb + tb;
              out[5 * count + 4] = (int32_t)mc + tc;
            }
            ++count;
            ++found;
          }
      if (found > 1) ++multi;
    }
  }
  if (several) *several = multi;
  return count;
}

/* The f32 pair test of a triclinic build, as the device computes it:
 * frames xw = (float)(x + S H), S the lattice vector that brings x into the
 * brick [0, ax) x [0, by) x [0, cz) (along c, then b, then a; in f64), the
 * image of an entry n in f32, t = n H with each product and sum rounded
 * (tx = (na ax + nb bx) + nc cx, ty = nb by + nc cy, tz = nc cz, the cell in
 * f32), and d = (xw_B + t) - xw_A, A the atom of the smaller number (t
 * negated when A is j); r2 = (dx dx + dy dy) + dz dz, no fused multiply-add;
 * the test r2 <= (float)(R'^2), R' the widened reach.  The images are those
 * of orc_pairset_triclinic's search (span lattice vectors from the reduced
 * image of the f64 displacement); rows (i, j, na, nb, nc) relative to the
 * raw positions. */
static void tri_wrap(const double *x, const double *cell, double *xw, int32_t *S) {
  double ax = cell[0], by = cell[1], cz = cell[2], bx = cell[3], cx = cell[4], cy = cell[5];
  double p[3] = {x[0], x[1], x[2]};
  double sc = -floor(p[2] / cz);
  p[0] += sc * cx; p[1] += sc * cy; p[2] += sc * cz;
  double sb = -floor(p[1] / by);
  p[0] += sb * bx; p[1] += sb * by;
  double sa = -floor(p[0] / ax);
  p[0] += sa * ax;
  xw[0] = p[0]; xw[1] = p[1]; xw[2] = p[2];
  S[0] = (int32_t)sa; S[1] = (int32_t)sb; S[2] = (int32_t)sc;
}

int64_t orc_pairset_triclinic_f32(int64_t n, const double *x, const double *cell, double reach,
                                  const int32_t *excl_off, const int32_t *excl, int32_t span, int64_t cap,
                                  int32_t *out) {
  float axf = (float)cell[0], byf = (float)cell[1], czf = (float)cell[2];
  float bxf = (float)cell[3], cxf = (float)cell[4], cyf = (float)cell[5];
  double ax = cell[0], by = cell[1], cz = cell[2], bx = cell[3], cx = cell[4], cy = cell[5];
  double Rw = orc_widened_reach_triclinic(reach, cell);
  float R2f = (float)(Rw * Rw);
  double Rs = Rw + 1e-3;  /* the f64 search reach of the candidate images */
  float *xf = (float *)malloc(sizeof(float) * 3 * (size_t)(n > 0 ? n : 1));
  double *xd = (double *)malloc(sizeof(double) * 3 * (size_t)(n > 0 ? n : 1));
  int32_t *S = (int32_t *)malloc(sizeof(int32_t) * 3 * (size_t)(n > 0 ? n : 1));
  for (int64_t i = 0; i < n; ++i) {
    if (!finite3(x + 3 * i)) continue;
    tri_wrap(x + 3 * i, cell, xd + 3 * i, S + 3 * i);
    for (int k = 0; k < 3; ++k) xf[3 * i + k] = (float)xd[3 * i + k];
  }
  int64_t count = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (!finite3(x + 3 * i)) continue;
    for (int64_t j = i + 1; j < n; ++j) {
      if (!finite3(x + 3 * j)) continue;
      if (excluded_pair(excl_off, excl, (int32_t)i, (int32_t)j)) continue;
      /* candidate images e of wrapped j relative to wrapped i */
      double d[3] = {xd[3 * j] - xd[3 * i], xd[3 * j + 1] - xd[3 * i + 1], xd[3 * j + 2] - xd[3 * i + 2]};
      double mc = -rint(d[2] / cz);
      d[0] += mc * cx; d[1] += mc * cy; d[2] += mc * cz;
      double mb = -rint(d[1] / by);
      d[0] += mb * bx; d[1] += mb * by;
      double ma = -rint(d[0] / ax);
      d[0] += ma * ax;
      for (int tc = -span; tc <= span; ++tc)
        for (int tb = -span; tb <= span; ++tb)
          for (int ta = -span; ta <= span; ++ta) {
            double ex = d[0] + ta * ax + tb * bx + tc * cx;
            double ey = d[1] + tb * by + tc * cy;
            double ez = d[2] + tc * cz;
            if (!(ex * ex + ey * ey + ez * ez <= Rs * Rs)) continue;
            int32_t na = (int32_t)ma + ta, nb = (int32_t)mb + tb, nc = (int32_t)mc + tc;
            /* the f32 test, A = i (the smaller number), B = j with image n */
            float fa = (float)na, fb = (float)nb, fc = (float)nc;
            float tx = (fa * axf + fb * bxf) + fc * cxf;
            float ty = fb * byf + fc * cyf;
            float tz = fc * czf;
            float dx = (xf[3 * j] + tx) - xf[3 * i];
            float dy = (xf[3 * j + 1] + ty) - xf[3 * i + 1];
            float dz = (xf[3 * j + 2] + tz) - xf[3 * i + 2];
            float r2 = (dx * dx + dy * dy) + dz * dz;
            if (!(r2 <= R2f)) continue;
            if (count < cap && out) {
              /* relative to the raw positions: n + S_j - S_i */
              out[5 * count] = (int32_t)i;
              out[5 * count + 1] = (int32_t)j;
              out[5 * count + 2] = na + S[3 * j] - S[3 * i];
              out[5 * count + 3] = nb + S[3 * j + 1] - S[3 * i + 1];
              out[5 * count + 4] = nc + S[3 * j + 2] - S[3 * i + 2];
            }
            ++count;
          }
    }
  }
  free(xf);
  free(xd);
  free(S);
  return count;
}

/* The Lennard-Jones + Ewald direct pair term of orc_nonbonded in a
 * triclinic cell: every image within rc of every pair i < j (the f64
 * displacement reduced once along c, b, a, then `span` lattice vectors
 * around it); small systems, O(n^2). */
void orc_nonbonded_triclinic(int64_t n, const double *x, const double *q, const int32_t *type, int32_t ntypes,
                             const double *sigma, const double *epsilon, const double *cell, double rc,
                             double beta, double coulomb, const int32_t *excl_off, const int32_t *excl,
                             int32_t span, double *forces, double *energies, double *virial) {
  double ax = cell[0], by = cell[1], cz = cell[2], bx = cell[3], cx = cell[4], cy = cell[5];
  double rc2 = rc * rc;
  double twobeta_sqrtpi = 2.0 * beta / sqrt(M_PI);
  double elj = 0.0, ecoul = 0.0, W[9] = {0};
  for (int64_t i = 0; i < n; ++i) {
    if (!finite3(x + 3 * i)) continue;
    for (int64_t j = i + 1; j < n; ++j) {
      if (!finite3(x + 3 * j)) continue;
      if (excluded_pair(excl_off, excl, (int32_t)i, (int32_t)j)) continue;
      double d0[3] = {x[3 * i] - x[3 * j], x[3 * i + 1] - x[3 * j + 1], x[3 * i + 2] - x[3 * j + 2]};
      double mc = -rint(d0[2] / cz);
      d0[0] += mc * cx; d0[1] += mc * cy; d0[2] += mc * cz;
      double mb = -rint(d0[1] / by);
      d0[0] += mb * bx; d0[1] += mb * by;
      d0[0] += -rint(d0[0] / ax) * ax;
      for (int tc = -span; tc <= span; ++tc)
        for (int tb = -span; tb <= span; ++tb)
          for (int ta = -span; ta <= span; ++ta) {
            double d[3] = {d0[0] + ta * ax + tb * bx + tc * cx, d0[1] + tb * by + tc * cy, d0[2] + tc * cz};
            double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            if (!(r2 < rc2)) continue;
            double r = sqrt(r2);
            double fscal = 0.0;
            int ti = type[i], tj = type[j];
            double sg = sigma[ti * ntypes + tj], ep = epsilon[ti * ntypes + tj];
            if (ep != 0.0) {
              double sr = sg / r, s6 = pow(sr, 6.0), s12 = s6 * s6;
              elj += 4.0 * ep * (s12 - s6);
              fscal += -(4.0 * ep * (-12.0 * s12 + 6.0 * s6) / r) / r;
            }
            double qq = coulomb * q[i] * q[j];
            if (qq != 0.0) {
              double er = erfc(beta * r);
              ecoul += qq * er / r;
              fscal += -(qq * (-er / r2 - twobeta_sqrtpi * exp(-beta * beta * r2) / r)) / r;
            }
            for (int k = 0; k < 3; ++k) {
              forces[3 * i + k] += fscal * d[k];
              forces[3 * j + k] -= fscal * d[k];
            }
            for (int a2 = 0; a2 < 3; ++a2)
              for (int b2 = 0; b2 < 3; ++b2) W[3 * a2 + b2] += d[a2] * fscal * d[b2];
          }
    }
  }
  energies[0] += elj;
  energies[1] += ecoul;
  for (int k = 0; k < 9; ++k) virial[k] += W[k];
}

/* orc_excluded in a triclinic cell: the minimum image reduced once along
 * c, b, a. */
void orc_excluded_triclinic(int64_t npairs, const int32_t *pairs, const double *x, const double *q,
                            const double *cell, double beta, double coulomb, double *forces, double *energies,
                            double *virial) {
  double ax = cell[0], by = cell[1], cz = cell[2], bx = cell[3], cx = cell[4], cy = cell[5];
  double e = 0.0;
  double twobeta_sqrtpi = 2.0 * beta / sqrt(M_PI);
  for (int64_t p = 0; p < npairs; ++p) {
    int32_t i = pairs[2 * p], j = pairs[2 * p + 1];
    double d[3] = {x[3 * i] - x[3 * j], x[3 * i + 1] - x[3 * j + 1], x[3 * i + 2] - x[3 * j + 2]};
    double mc = -rint(d[2] / cz);
    d[0] += mc * cx; d[1] += mc * cy; d[2] += mc * cz;
    double mb = -rint(d[1] / by);
    d[0] += mb * bx; d[1] += mb * by;
    d[0] += -rint(d[0] / ax) * ax;
    double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    double qq = coulomb * q[i] * q[j];
    if (qq == 0.0 || r2 <= 0.0) continue;
    double r = sqrt(r2);
    double ef = erf(beta * r);
    e += -qq * ef / r;
    double fs = qq * (twobeta_sqrtpi * exp(-beta * beta * r2) / r2 - ef / (r2 * r));
    for (int k = 0; k < 3; ++k) {
      forces[3 * i + k] += fs * d[k];
      forces[3 * j + k] -= fs * d[k];
    }
    for (int a2 = 0; a2 < 3; ++a2)
      for (int b2 = 0; b2 < 3; ++b2) virial[3 * a2 + b2] += d[a2] * fs * d[b2];
  }
  energies[0] += e;
}
