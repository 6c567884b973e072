// The MD step around the nonbonded + PME term, on sm_100a: leap-frog with
// SETTLE for rigid waters, the Bussi (CSVR) thermostat, and MDIR's exact
// test of validity of the lists (D80), all on the device, captured as one
// CUDA graph of `unroll` steps whose rebuild of the lists is a conditional
// node set by the device itself (no host round trip per step).
//
// MDIR's step (docs/dynamics.md; docs/neighbor-groups.md, Sections 1.4 and
// 7.1; runtime/mdrt_step_graph.cu for the idea of a replayed step) keeps
// water rigid by M-SHAKE below double precision (D112); SETTLE
// (Miyamoto & Kollman, J. Comput. Chem. 13 (1992) 952) is the analytic
// solution of the same constraints for a rigid three-site water.
//
// One step (B200 design):
//   fork:  PME (spread, R2C, convolve, C2R, gather) on a high-priority side
//          stream  ||  pair kernel (+ excluded pairs outside waters)
//   join:  md_update, a thread per water: reads the place accumulators of its
//          three atoms (pairs + PME), adds the three intra-water excluded
//          Ewald corrections in f64, integrates, applies SETTLE, writes x, v,
//          the f32 frames of the next step and clears the accumulators
//          md_thermostat: kinetic energy (fixed-order f64), Bussi scaling, and
//          the test of validity that sets the conditional rebuild
//   if rebuild: the neighbor build, the frames, the reference positions
#include <cmath>
#include <cstring>
#include <cstdio>
#include <vector>

#include "../../include/mdrt_nb.h"
#include "nb_context.h"
#include "nb_spline.cuh"

#define MD_MAX_UNROLL 256  // steps of one replayed graph
#define MD_CK(x)                                      \
  do {                                                \
    if ((x) != cudaSuccess) return MDRT_NB_CUDA_ERROR; \
  } while (0)
#define MD_IN_FLIGHT 2     // step graphs queued ahead of the one the host checks

struct mdrtMd {
  NbCtx *nb = nullptr;
  mdrtNb *handle = nullptr;
  int device = 0;                  // the context's device (the context may go first)
  int64_t n = 0, nwaters = 0, nfree = 0;
  double *inv_mass = nullptr;      // device f64 [n]
  double *mass = nullptr;          // device f64 [n]
  int32_t *waters = nullptr;       // device [nw][3] (O, H1, H2)
  int32_t *free_atoms = nullptr;   // device [nfree]
  int32_t *excl_other = nullptr;   // excluded pairs not inside one water (i < j)
  int64_t n_excl_other = 0;
  bool water_excl = false;         // the three pairs of each water are excluded
  double dOH = 0.09572, dHH = 0.15139, mO = 15.9994, mH = 1.008;
  double *force = nullptr;         // device f64 [n, 3]: the forces of the last step
  double *x_ref = nullptr;         // positions at the last build
  double *x_prune = nullptr;       // positions at the last pruning (dual list)
  double *ke_part = nullptr;       // per-block kinetic partials
  int ke_blocks = 0;
  unsigned int *done_blocks = nullptr;  // blocks of md_update finished (the last one reduces)
  float2 *blk_max = nullptr;       // per block of md_update: max |x - x_ref|^2, max |x - x_prune|^2
  unsigned int *drift = nullptr;   // mdrtMdRefresh: the same two maxima of a new state (f32 bits)
  int32_t *wplace = nullptr;       // the place of each water atom, by slot 3 w + k (after each build)
  int32_t *fplace = nullptr;       // the place of each free atom, by its slot
  double *thermo = nullptr;        // [0] lambda, [1] KE, [2] KE before, [3] steps, [4] builds, [5] prunes
  double *noise = nullptr;         // thermostat draws of the steps of one launch (2 a step)
  int *flag = nullptr;             // [0] rebuild, [1] prune: flags for the step-by-step path
  // The checkpoint of a run of step graphs (positions, velocities, thermo)
  // and what its builds saw: [0] the longest list, [1] capacity overflow
  // bits, [2] builds that met positions that are not finite.
  double *x_ck = nullptr, *v_ck = nullptr, *thermo_ck = nullptr;
  double *xref_ck = nullptr, *xprune_ck = nullptr;  // the reference positions of the lists in force
  int32_t *peak = nullptr, *h_peak = nullptr;
  double *h_steps = nullptr;       // pinned: the step counter at the checkpoint and after the run
  int64_t regrows = 0;             // runs redone after an overflow inside the graphs
  int64_t redone = 0;              // stops at a drift past half the skin between two decisions
  double lookahead = 1.5;          // mdrtMdSetLookahead
  int verlet = 0;                  // mdrtMdSetIntegrator: velocities on the step at a run's ends
  // PME gathered by the update (order 4): the step's side stream spreads the
  // frames into qgrid (through qfixed in the deterministic mode) and
  // transforms qgrid -> spec -> phi; the update gathers each atom's PME force
  float *qgrid = nullptr, *phi = nullptr;
  unsigned long long *qfixed = nullptr;
  float2 *spec = nullptr;
  float *influence = nullptr;      // B C, f32 per half-complex point, of influence_key
  double influence_key[7] = {0, 0, 0, 0, 0, 0, 0};  // cell, beta, f, grid
  int64_t pme_points = 0;          // K0 K1 K2 the buffers were sized for
  // A stop at a stale list, seen by the host while step graphs are queued:
  // the update writes 1 into mapped pinned memory, and the host, which keeps
  // at most MD_IN_FLIGHT graphs queued beyond the one it waits for, stops
  // launching (the graphs after a stop would do nothing).
  int *h_halt = nullptr, *d_halt = nullptr;
  cudaEvent_t ev_run[MD_IN_FLIGHT + 1] = {};
  double temperature = 300.0, tau = 0.0;
  int64_t ndof = 0;
  unsigned long long seed = 1;
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // graph
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;
  const double *gx = nullptr, *gv = nullptr;
  double gbox[3] = {0, 0, 0};
  double gdt = 0.0;
  int gunroll = 0;
  int64_t gcap_key = -1;
  std::vector<cudaGraphConditionalHandle> handles;
};

namespace {

struct Vec3 {
  double x, y, z;
};
__device__ __forceinline__ Vec3 operator-(Vec3 a, Vec3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ Vec3 operator+(Vec3 a, Vec3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ Vec3 operator*(double s, Vec3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ double dot(Vec3 a, Vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ Vec3 cross(Vec3 a, Vec3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ Vec3 unit(Vec3 a) { return rsqrt(dot(a, a)) * a; }
__device__ __forceinline__ Vec3 load3(const double *p, int64_t i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
__device__ __forceinline__ void store3(double *p, int64_t i, Vec3 v) {
  p[3 * i] = v.x;
  p[3 * i + 1] = v.y;
  p[3 * i + 2] = v.z;
}

struct SettleParams {
  double mO, mH, ra, rb, rc;  // canonical triangle: O at ra from the centre of mass, H pair at rb, half HH rc
};

// SETTLE: the constrained positions of one water from its constrained old
// positions a0, b0, c0 and unconstrained new a1, b1, c1 (overwritten).
__device__ void settle(const SettleParams &P, Vec3 a0, Vec3 b0, Vec3 c0, Vec3 &a1, Vec3 &b1, Vec3 &c1) {
  double M = P.mO + 2.0 * P.mH;
  Vec3 d = (1.0 / M) * (P.mO * a1 + P.mH * b1 + P.mH * c1);  // centre of mass of the new positions
  Vec3 A1 = a1 - d, B1 = b1 - d, C1 = c1 - d;
  Vec3 B0 = b0 - a0, C0 = c0 - a0;
  Vec3 ez = unit(cross(B0, C0));  // normal of the old plane
  Vec3 ex = unit(cross(A1, ez));  // perpendicular to it and to the new O
  Vec3 ey = cross(ez, ex);
  double xb0 = dot(B0, ex), yb0 = dot(B0, ey);
  double xc0 = dot(C0, ex), yc0 = dot(C0, ey);
  double za1 = dot(A1, ez);
  double xb1 = dot(B1, ex), yb1 = dot(B1, ey), zb1 = dot(B1, ez);
  double xc1 = dot(C1, ex), yc1 = dot(C1, ey), zc1 = dot(C1, ez);
  double sinphi = za1 / P.ra;
  double cosphi = sqrt(fmax(0.0, 1.0 - sinphi * sinphi));
  double sinpsi = (zb1 - zc1) / (2.0 * P.rc * cosphi);
  double cospsi = sqrt(fmax(0.0, 1.0 - sinpsi * sinpsi));
  double ya2 = P.ra * cosphi;
  double xb2 = -P.rc * cospsi;
  double yb2 = -P.rb * cosphi - P.rc * sinpsi * sinphi;
  double yc2 = -P.rb * cosphi + P.rc * sinpsi * sinphi;
  double alpha = xb2 * (xb0 - xc0) + yb0 * yb2 + yc0 * yc2;
  double beta = xb2 * (yc0 - yb0) + xb0 * yb2 + xc0 * yc2;
  double gamma = xb0 * yb1 - xb1 * yb0 + xc0 * yc1 - xc1 * yc0;
  double ab2 = alpha * alpha + beta * beta;
  double sintheta = (alpha * gamma - beta * sqrt(fmax(0.0, ab2 - gamma * gamma))) / ab2;
  double costheta = sqrt(fmax(0.0, 1.0 - sintheta * sintheta));
  double xa3 = -ya2 * sintheta, ya3 = ya2 * costheta;
  double xb3 = xb2 * costheta - yb2 * sintheta, yb3 = xb2 * sintheta + yb2 * costheta;
  double xc3 = -xb2 * costheta - yc2 * sintheta, yc3 = -xb2 * sintheta + yc2 * costheta;
  a1 = d + (xa3 * ex + ya3 * ey + za1 * ez);
  b1 = d + (xb3 * ex + yb3 * ey + zb1 * ez);
  c1 = d + (xc3 * ex + yc3 * ey + zc1 * ez);
}

struct UpdateParams {
  SettleParams S;
  double dt;
  double L[3];
  double beta, coulomb, two_beta_sqrtpi;
  int water_excl;
  int fixed;
  // thermostat and the tests of validity, done by the last block
  double tau, temperature, ndof;
  double build_half2, prune_half2;  // ((R - r_c)/2)^2 and ((R_in - r_c)/2)^2 (0: no dual list)
  cudaGraphConditionalHandle h_any;  // the step's conditional node: a rebuild or a pruning is due
  int use_graph;
  int *flag;  // [0] rebuild, [1] prune (device)
  const double *noise;  // the thermostat's draws of the steps of this launch
  int k;                // this step's index among them
  // the rebuild is decided ahead, at the last step of each window of steps
  // (check_build), from the drift and its growth over the window; at the
  // other steps a drift past half the skin marks the lists stale (status),
  // and the run is redone
  int check_build;
  double lookahead;  // the growth of the last window extrapolated this many times
  int *status;
  int32_t *peak;
  // PME inside the update (order 4): the potential to gather from (0: the
  // PME forces come in `pme`)
  int pme_fused;
  GridParams G;
  const float *phi;
  int *host_halt;  // mapped pinned memory: 1 when a stale list stopped the steps
  int32_t *unit_counter;  // zeroed with a pruning due: the pruning's blocks claim their units from it
};

// The force on atom a: the pair / excluded accumulator of its place and the
// PME force; clears the accumulator for the next step.
__device__ __forceinline__ Vec3 take_force(int p, float4 *acc, unsigned long long *accf,
                                           const float4 *__restrict__ pme, int fixed) {
  if (p < 0) return {0.0, 0.0, 0.0};
  Vec3 f;
  if (fixed) {
    long long x = (long long)accf[3 * p], y = (long long)accf[3 * p + 1], z = (long long)accf[3 * p + 2];
    accf[3 * p] = 0ull;
    accf[3 * p + 1] = 0ull;
    accf[3 * p + 2] = 0ull;
    f = {(double)x * NB_FORCE_SCALE_INV, (double)y * NB_FORCE_SCALE_INV, (double)z * NB_FORCE_SCALE_INV};
  } else {
    float4 v = acc[p];
    acc[p] = make_float4(0.f, 0.f, 0.f, 0.f);
    f = {v.x, v.y, v.z};
  }
  if (pme) {
    float4 w = pme[p];
    f.x += w.x;
    f.y += w.y;
    f.z += w.z;
  }
  return f;
}

// The frame of place p at x (the charge kept), and with xq_lo its f32
// residual (the split frames of the deterministic mode).
__device__ __forceinline__ float4 md_frame(int p, Vec3 x, char4 s, const double *L, float q, float4 *xq,
                                           float4 *xq_lo) {
  // rounded as nb_gather rounds the frames of a build (no contraction)
  double fx = __dadd_rn(x.x, __dmul_rn(nb_frame_shift(s.x), L[0]));
  double fy = __dadd_rn(x.y, __dmul_rn(nb_frame_shift(s.y), L[1]));
  double fz = __dadd_rn(x.z, __dmul_rn(nb_frame_shift(s.z), L[2]));
  float4 nf = make_float4((float)fx, (float)fy, (float)fz, q);
  xq[p] = nf;
  if (xq_lo)
    xq_lo[p] = make_float4((float)(fx - (double)nf.x), (float)(fy - (double)nf.y), (float)(fz - (double)nf.z), 0.f);
  return nf;
}

__device__ __forceinline__ float4 write_frame(int p, Vec3 x, const char4 *__restrict__ shift, const double *L,
                                              float4 *xq, float4 *xq_lo) {
  if (p < 0) return make_float4(0.f, 0.f, 0.f, 0.f);
  return md_frame(p, x, shift[p], L, xq[p].w, xq, xq_lo);
}

// The PME force on the atom at frame fr (charge fr.w), gathered from the
// potential grid with order-4 B-splines: F = -q sum_k phi(k) grad W(k).
__device__ __forceinline__ Vec3 md_pme_gather(float4 fr, const float *__restrict__ phi, const GridParams &G) {
  int k0, k1, k2;
  float t0, t1, t2;
  nb_frac(fr.x, G.invL0, G.K0, k0, t0);
  nb_frac(fr.y, G.invL1, G.K1, k1, t1);
  nb_frac(fr.z, G.invL2, G.K2, k2, t2);
  float w0[4], w1[4], w2[4], d0[4], d1[4], d2[4];
  nb_bspline<4>(t0, w0, d0);
  nb_bspline<4>(t1, w1, d1);
  nb_bspline<4>(t2, w2, d2);
  int gzs[4];
#pragma unroll
  for (int jz = 0; jz < 4; ++jz) {
    int gz = k2 - jz;
    gzs[jz] = gz < 0 ? gz + G.K2 : gz;
  }
  float g0 = 0.f, g1 = 0.f, g2 = 0.f;
#pragma unroll
  for (int jx = 0; jx < 4; ++jx) {
    int gx = k0 - jx;
    if (gx < 0) gx += G.K0;
#pragma unroll
    for (int jy = 0; jy < 4; ++jy) {
      int gy = k1 - jy;
      if (gy < 0) gy += G.K1;
      const float *row = phi + ((int64_t)gx * G.K1 + gy) * G.K2;
      float sz = 0.f, sdz = 0.f;
#pragma unroll
      for (int jz = 0; jz < 4; ++jz) {
        float f = __ldg(row + gzs[jz]);
        sz = fmaf(f, w2[jz], sz);
        sdz = fmaf(f, d2[jz], sdz);
      }
      g0 = fmaf(d0[jx] * w1[jy], sz, g0);
      g1 = fmaf(w0[jx] * d1[jy], sz, g1);
      g2 = fmaf(w0[jx] * w1[jy], sdz, g2);
    }
  }
  float q = fr.w;
  return {(double)(-q * g0 * (float)G.K0 * G.invL0), (double)(-q * g1 * (float)G.K1 * G.invL1),
          (double)(-q * g2 * (float)G.K2 * G.invL2)};
}

#define MD_UPDATE_THREADS 64

__device__ void md_last_block(const UpdateParams &U, const double *ke_part, const float2 *blk_max, int nblocks,
                              double *thermo, unsigned int *counter);

__device__ __forceinline__ Vec3 shfl3(Vec3 a, int src) {
  return {__shfl_sync(0xffffffffu, a.x, src), __shfl_sync(0xffffffffu, a.y, src), __shfl_sync(0xffffffffu, a.z, src)};
}

// One leap-frog step with SETTLE: v = lambda v + f/m dt; x += v dt;
// constrain; v = (x_new - x_old)/dt.
//
// Waters: a lane per atom, three neighbouring lanes per water (10 waters a
// warp, lanes 30 and 31 idle), so that the loads of every atom are issued
// at once and coalesced: the step is bound by two memory round trips (the
// place of the atom, then its accumulators), not by a chain of them.  Lane k
// of a water computes the excluded Ewald correction of the pair (k, k+1) in
// f64, the lanes exchange positions and forces by shuffles, and each
// evaluates SETTLE for its water (the same inputs, so the same result) and
// writes its own atom.  Blocks past the waters take the free atoms, a thread
// each.  The last block to finish sums the kinetic energy in a fixed order
// and runs the thermostat and the tests of validity (md_last_block).
__global__ void __launch_bounds__(MD_UPDATE_THREADS) md_update(
    int64_t nwaters, int64_t nfree, const int32_t *__restrict__ waters, const int32_t *__restrict__ free_atoms,
    UpdateParams U, const double *__restrict__ inv_mass, const double *__restrict__ mass,
    const float *__restrict__ charge, const int32_t *__restrict__ wplace, const int32_t *__restrict__ fplace,
    const char4 *__restrict__ shift, float4 *acc, unsigned long long *accf, const float4 *__restrict__ pme,
    float4 *xq, float4 *xq_lo, double *__restrict__ x, double *__restrict__ v, double *__restrict__ fout,
    const double *__restrict__ x_ref, const double *__restrict__ x_prune, double *thermo, double *ke_part,
    float2 *blk_max, unsigned int *counter) {
  __shared__ double s_ke[MD_UPDATE_THREADS / 32];
  __shared__ float s_d2[MD_UPDATE_THREADS / 32], s_p2[MD_UPDATE_THREADS / 32];
  __shared__ int s_last;
  // read beside the first loads; the state stays at a step that a stale list stopped
  const int halt = U.flag[3];
  const int WPB = MD_UPDATE_THREADS / 32 * 10;  // waters per block
  int64_t water_blocks = (nwaters + WPB - 1) / WPB;
  double lambda = thermo[0];
  double dt = U.dt;
  double ke = 0.0;
  float d2max = 0.f, p2max = 0.f;
  if (blockIdx.x < water_blocks) {
    int lane = threadIdx.x & 31, wl = lane / 3, k = lane - 3 * (lane / 3);
    int64_t w = ((int64_t)blockIdx.x * (MD_UPDATE_THREADS / 32) + (threadIdx.x >> 5)) * 10 + wl;
    bool act = lane < 30 && w < nwaters;
    // the atom and its place, both by the water's slot: one memory round
    // trip before the loads by atom and by place
    int a = act ? waters[3 * w + k] : 0;
    int p = act ? wplace[3 * w + k] : -1;
    int base = 3 * wl, s1 = base + (k + 1) % 3, s2 = base + (k + 2) % 3;
    if (lane >= 30) s1 = s2 = base = lane;
    // every load of data that no kernel of this step writes (the pair
    // kernel lets this launch start beside it, so the step's pruning may not
    // have flushed), then the wait
    Vec3 x0 = load3(x, a), v0 = load3(v, a);
    double q = charge[a], im = inv_mass[a], ms = mass[a];
    Vec3 xr = load3(x_ref, a);
    char4 sh = p >= 0 ? shift[p] : make_char4(0, 0, 0, 0);
    float4 fr = p >= 0 ? xq[p] : make_float4(0.f, 0.f, 0.f, 0.f);
    float qw = p >= 0 ? fr.w : 0.f;
    // the PME gather (the potential comes from the reciprocal chain, which
    // the launch depends on in full) and the excluded pair (k, k+1) of this
    // water (positions only) need nothing of the pair kernel: both run
    // before the wait, beside that kernel's last units
    Vec3 fg = {0.0, 0.0, 0.0};
    if (p >= 0 && U.pme_fused && qw != 0.f) fg = md_pme_gather(fr, U.phi, U.G);
    Vec3 x1 = shfl3(x0, s1);
    double q1 = __shfl_sync(0xffffffffu, q, s1);
    Vec3 fp = {0.0, 0.0, 0.0};
    if (U.water_excl && act) {
      Vec3 d = x0 - x1;
      d.x -= U.L[0] * rint(d.x / U.L[0]);
      d.y -= U.L[1] * rint(d.y / U.L[1]);
      d.z -= U.L[2] * rint(d.z / U.L[2]);
      double r2 = dot(d, d), qq = U.coulomb * q * q1;
      if (qq != 0.0 && r2 > 0.0) {
        double r = sqrt(r2);
        double fs = qq * (U.two_beta_sqrtpi * exp(-U.beta * U.beta * r2) / r2 - erf(U.beta * r) / (r2 * r));
        fp = fs * d;
      }
    }
    nb_grid_wait();
    if (halt) return;
    // the positions of the last pruning: a pruning of this step (before the
    // pair kernel) writes them
    Vec3 xpr = U.prune_half2 > 0.0 ? load3(x_prune, a) : xr;
    Vec3 f = {0.0, 0.0, 0.0};
    if (p >= 0) {
      if (U.fixed) {
        long long fx = (long long)accf[3 * p], fy = (long long)accf[3 * p + 1], fz = (long long)accf[3 * p + 2];
        f = {(double)fx * NB_FORCE_SCALE_INV, (double)fy * NB_FORCE_SCALE_INV, (double)fz * NB_FORCE_SCALE_INV};
      } else {
        float4 f4 = acc[p];
        f = {f4.x, f4.y, f4.z};
      }
      if (pme) {
        float4 w4 = pme[p];
        f.x += w4.x;
        f.y += w4.y;
        f.z += w4.z;
      }
      if (U.pme_fused && qw != 0.f) {
        f.x += fg.x;
        f.y += fg.y;
        f.z += fg.z;
      }
    }
    // this atom: + its own pair, - the pair (k-1, k) of the lane before
    f = f + fp - shfl3(fp, s2);
    // the three atoms of the water, in O, H, H order
    Vec3 xa = shfl3(x0, base), xb = shfl3(x0, base + 1), xc = shfl3(x0, base + 2);
    Vec3 va = shfl3(v0, base), vb = shfl3(v0, base + 1), vc = shfl3(v0, base + 2);
    Vec3 fa = shfl3(f, base), fb = shfl3(f, base + 1), fc = shfl3(f, base + 2);
    double ima = __shfl_sync(0xffffffffu, im, base), imb = __shfl_sync(0xffffffffu, im, base + 1),
           imc = __shfl_sync(0xffffffffu, im, base + 2);
    va = lambda * va + (dt * ima) * fa;
    vb = lambda * vb + (dt * imb) * fb;
    vc = lambda * vc + (dt * imc) * fc;
    Vec3 a1 = xa + dt * va, b1 = xb + dt * vb, c1 = xc + dt * vc;
    settle(U.S, xa, xb, xc, a1, b1, c1);
    Vec3 xn = k == 0 ? a1 : (k == 1 ? b1 : c1);
    if (act) {
      Vec3 vn = (1.0 / dt) * (xn - x0);
      store3(x, a, xn);
      store3(v, a, vn);
      store3(fout, a, f);
      if (p >= 0) {
        md_frame(p, xn, sh, U.L, qw, xq, xq_lo);
        if (U.fixed) {
          accf[3 * p] = 0ull;
          accf[3 * p + 1] = 0ull;
          accf[3 * p + 2] = 0ull;
        } else {
          acc[p] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
      }
      ke = 0.5 * ms * dot(vn, vn);
      Vec3 dr = xn - xr;
      d2max = (float)dot(dr, dr);
      if (U.prune_half2 > 0.0) {
        dr = xn - xpr;
        p2max = (float)dot(dr, dr);
      }
    }
  } else if ((int64_t)(blockIdx.x - water_blocks) * blockDim.x + threadIdx.x < nfree) {
    int64_t t = (int64_t)(blockIdx.x - water_blocks) * blockDim.x + threadIdx.x;
    int i = free_atoms[t];
    int pi = fplace[t];
    Vec3 fg = {0.0, 0.0, 0.0};
    bool gather = false;
    if (U.pme_fused && pi >= 0) {
      float4 fr = xq[pi];
      gather = fr.w != 0.f;
      if (gather) fg = md_pme_gather(fr, U.phi, U.G);
    }
    nb_grid_wait();
    if (halt) return;
    Vec3 fi = take_force(pi, acc, accf, pme, U.fixed);
    if (gather) fi = fi + fg;
    Vec3 vi = lambda * load3(v, i) + (dt * inv_mass[i]) * fi;
    Vec3 xi = load3(x, i) + dt * vi;
    store3(x, i, xi);
    store3(v, i, vi);
    store3(fout, i, fi);
    write_frame(pi, xi, shift, U.L, xq, xq_lo);
    ke = 0.5 * mass[i] * dot(vi, vi);
    Vec3 di = xi - load3(x_ref, i);
    d2max = (float)dot(di, di);
    if (U.prune_half2 > 0.0) {
      di = xi - load3(x_prune, i);
      p2max = (float)dot(di, di);
    }
  }
  nb_grid_wait();
  if (halt) return;  // every thread of the grid, the idle ones too: no barrier is reached
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ke += __shfl_xor_sync(0xffffffffu, ke, o);
    d2max = fmaxf(d2max, __shfl_xor_sync(0xffffffffu, d2max, o));
    p2max = fmaxf(p2max, __shfl_xor_sync(0xffffffffu, p2max, o));
  }
  if (lane == 0) {
    s_ke[warp] = ke;
    s_d2[warp] = d2max;
    s_p2[warp] = p2max;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    float m = 0.f, mp = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      s += s_ke[w];
      m = fmaxf(m, s_d2[w]);
      mp = fmaxf(mp, s_p2[w]);
    }
    ke_part[blockIdx.x] = s;
    blk_max[blockIdx.x] = make_float2(m, mp);  // no contended atomics: the last block reduces them
    __threadfence();
    unsigned done = atomicAdd(counter, 1u);
    s_last = done == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last) md_last_block(U, ke_part, blk_max, gridDim.x, thermo, counter);
}

// splitmix64 (Steele, Lea & Flood 2014) as a counter-based generator.
__device__ __forceinline__ unsigned long long splitmix(unsigned long long z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ double uniform01(unsigned long long &ctr, unsigned long long seed) {
  unsigned long long r = splitmix(seed ^ splitmix(ctr++));
  return ((r >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}
__device__ __forceinline__ double normal01(unsigned long long &ctr, unsigned long long seed) {
  double u1 = uniform01(ctr, seed), u2 = uniform01(ctr, seed);
  return sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
}
// Gamma(a, 1), a >= 1, by Marsaglia & Tsang (ACM TOMS 26 (2000) 363); the
// loop is bounded and falls back to the mean.
__device__ double gamma_draw(double a, unsigned long long &ctr, unsigned long long seed) {
  double d = a - 1.0 / 3.0, c = 1.0 / sqrt(9.0 * d);
  for (int it = 0; it < 64; ++it) {
    double z = normal01(ctr, seed);
    double w = 1.0 + c * z;
    if (w <= 0.0) continue;
    w = w * w * w;
    double u = uniform01(ctr, seed);
    if (u < 1.0 - 0.0331 * z * z * z * z) return d * w;
    if (log(u) < 0.5 * z * z + d * (1.0 - w + log(w))) return d * w;
  }
  return a;
}

// The noise of the Bussi thermostat for the next `count` steps, a thread
// per step: a normal R1 and the sum of ndof - 1 squared normals
// (2 Gamma((ndof - 1)/2)), from the step counter and the seed, so that a
// step draws the same numbers however the steps are launched.  One launch
// at the head of a replayed graph serves all its steps.
__global__ void md_noise(const double *thermo, double *noise, int count, double ndof, unsigned long long seed) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  unsigned long long ctr = ((unsigned long long)thermo[3] + (unsigned long long)k) * 1024ull;
  noise[2 * k] = normal01(ctr, seed);
  noise[2 * k + 1] = ndof > 1.0 ? 2.0 * gamma_draw(0.5 * (ndof - 1.0), ctr, seed) : 0.0;
}

// The last block of md_update: the kinetic energy of the half step
// (fixed-order f64 sum), the Bussi (CSVR; Bussi, Donadio & Parrinello,
// J. Chem. Phys. 126 (2007) 014101) scaling for the next update, and the
// tests of validity (D80 and D114, the cell unchanged):
// rebuild when 2 max|x - x_build| > R - r_c, prune when rebuilt or
// 2 max|x - x_prune| > R_in - r_c; they set the conditional nodes.
__device__ void md_last_block(const UpdateParams &U, const double *ke_part, const float2 *blk_max, int nblocks,
                              double *thermo, unsigned int *counter) {
  __shared__ double s_k[MD_UPDATE_THREADS / 32];
  __shared__ float s_m[MD_UPDATE_THREADS / 32][2];
  double v = 0.0;
  float dmax = 0.f, pmax = 0.f;
  // eight partials a thread in flight at a time, summed in the order of b
  constexpr int CH = 8;
  for (int b0 = threadIdx.x; b0 < nblocks; b0 += CH * blockDim.x) {
    double kp[CH];
    float2 mb[CH];
#pragma unroll
    for (int r = 0; r < CH; ++r) {
      int b = b0 + r * blockDim.x;
      kp[r] = b < nblocks ? __ldcg(ke_part + b) : 0.0;
      mb[r] = b < nblocks ? __ldcg(blk_max + b) : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int r = 0; r < CH; ++r) {
      if (b0 + r * (int)blockDim.x < nblocks) v += kp[r];
      dmax = fmaxf(dmax, mb[r].x);
      pmax = fmaxf(pmax, mb[r].y);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v += __shfl_xor_sync(0xffffffffu, v, o);
    dmax = fmaxf(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
    pmax = fmaxf(pmax, __shfl_xor_sync(0xffffffffu, pmax, o));
  }
  if ((threadIdx.x & 31) == 0) {
    s_k[threadIdx.x >> 5] = v;
    s_m[threadIdx.x >> 5][0] = dmax;
    s_m[threadIdx.x >> 5][1] = pmax;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  double K = 0.0;
  float d2 = 0.f, p2 = 0.f;
  for (int w = 0; w < MD_UPDATE_THREADS / 32; ++w) {
    K += s_k[w];
    d2 = fmaxf(d2, s_m[w][0]);
    p2 = fmaxf(p2, s_m[w][1]);
  }
  thermo[2] = thermo[1];
  thermo[1] = K;
  thermo[3] += 1.0;
  double lambda = 1.0;
  if (U.tau > 0.0 && K > 0.0 && U.ndof > 1.0) {
    const double kB = 0.0083144626181532;
    double Kt = 0.5 * U.ndof * kB * U.temperature;
    double c = exp(-U.dt / U.tau);
    double r1 = U.noise[2 * U.k], sum = U.noise[2 * U.k + 1];
    double Knew = K + (1.0 - c) * (Kt * (r1 * r1 + sum) / U.ndof - K) + 2.0 * r1 * sqrt(c * (1.0 - c) * K * Kt / U.ndof);
    lambda = sqrt(fmax(Knew, 0.0) / K);
  }
  thermo[0] = lambda;
  int stale = (double)d2 > U.build_half2 ? 1 : 0;
  int rebuild = 0;
  if (U.check_build) {
    // the drift the lists may reach before the next decision: its growth
    // over the window just ended, once more (thermo[6] holds the drift at
    // the last decision, 0 after a build; the largest drift grows slower
    // than the first, ballistic, window); a wrong guess is caught by the test
    // of every step and costs a redo, not a missed pair
    double d = sqrt((double)d2);
    double ahead = d + U.lookahead * fmax(d - thermo[6], 0.0) + 0.002;
    rebuild = (stale || ahead * ahead > U.build_half2) ? 1 : 0;
    thermo[6] = d;
    stale = 0;
  }
  if (stale && U.use_graph) {
    // the lists of the next step are not sure: the steps after this one do
    // nothing (flag[3]), and the host rebuilds here and runs the rest
    atomicOr(U.status, NB_STATUS_STALE_LIST);
    atomicAdd(&U.peak[3], 1);
    U.flag[3] = 1;
    if (U.host_halt) *(volatile int *)U.host_halt = 1;
  }
  int prune = (U.prune_half2 > 0.0 && (rebuild || (double)p2 > U.prune_half2)) ? 1 : 0;
  // the host's build after a stale list (or, step by step, after a rebuild) prunes too
  if (stale || (!U.use_graph && rebuild)) prune = 0;
  *counter = 0u;
  U.flag[0] = rebuild;
  U.flag[1] = prune;
  if (prune && U.unit_counter) *U.unit_counter = 0;
  U.flag[2] = stale;
  if (U.use_graph && U.check_build) cudaGraphSetConditional(U.h_any, rebuild);
}

// After a build: the place of every atom by its slot in the integrator's
// lists (waters 3 w + k, then the free atoms), which md_update reads beside
// the slots' atom numbers instead of after them.
__global__ void md_places(int64_t nw3, int64_t nfree, const int32_t *__restrict__ waters,
                          const int32_t *__restrict__ free_atoms, const int32_t *__restrict__ place_of,
                          int32_t *__restrict__ wplace, int32_t *__restrict__ fplace) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nw3)
    wplace[k] = place_of[waters[k]];
  else if (k - nw3 < nfree)
    fplace[k - nw3] = place_of[free_atoms[k - nw3]];
}

// After a build: the reference positions, the counters, and what the build
// saw (the longest list, overflow, positions that are not finite), for the
// host check at the end of a run of step graphs.
__global__ void md_after_build(int64_t n3, const double *__restrict__ x, double *__restrict__ x_ref,
                               double *thermo, const int32_t *sizes, int *status, int32_t *peak) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n3) x_ref[k] = x[k];
  if (k == 0) {
    thermo[4] += 1.0;
    thermo[6] = 0.0;  // the drift at the last rebuild decision
    atomicMax(&peak[0], sizes[NB_SIZE_LONGEST]);
    if (sizes[NB_SIZE_OVERFLOW] != 0) {
      atomicOr(status, NB_STATUS_LIST_OVERFLOW);
      atomicOr(&peak[1], sizes[NB_SIZE_OVERFLOW]);
    }
    if (sizes[NB_SIZE_NAN] != 0) {
      atomicOr(status, NB_STATUS_NAN);
      atomicAdd(&peak[2], 1);
    }
  }
}

__global__ void md_clear_status(int *status, int bits) { atomicAnd(status, ~bits); }

// The largest squared drift of x from the positions of the last build and
// of the last pruning, each rounded to f32 as the update rounds its own
// (the bits of non-negative floats order as the floats): out[0], out[1].
__global__ void md_drift(int64_t n, const double *__restrict__ x, const double *__restrict__ x_ref,
                         const double *__restrict__ x_prune, unsigned int *out) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  float d2 = 0.f, p2 = 0.f;
  if (i < n) {
    Vec3 xi = load3(x, i);
    Vec3 dr = xi - load3(x_ref, i);
    d2 = (float)dot(dr, dr);
    if (x_prune) {
      dr = xi - load3(x_prune, i);
      p2 = (float)dot(dr, dr);
    }
    // a coordinate that is not finite counts as beyond any skin
    if (!(d2 <= 3.0e38f)) d2 = 3.0e38f;
    if (!(p2 <= 3.0e38f)) p2 = 3.0e38f;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    d2 = fmaxf(d2, __shfl_xor_sync(0xffffffffu, d2, o));
    p2 = fmaxf(p2, __shfl_xor_sync(0xffffffffu, p2, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(out, __float_as_uint(d2));
    atomicMax(out + 1, __float_as_uint(p2));
  }
}

// After a pruning: the reference positions of the inner list.
__global__ void md_after_prune(int64_t n3, const double *__restrict__ x, double *__restrict__ x_prune,
                               double *thermo) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n3) x_prune[k] = x[k];
  if (k == 0) thermo[5] += 1.0;
}

inline int blocks_for(int64_t n, int t) { return (int)std::max<int64_t>(1, (n + t - 1) / t); }

}  // namespace

static SettleParams settle_params(const mdrtMd &m) {
  SettleParams S;
  S.mO = m.mO;
  S.mH = m.mH;
  S.rc = 0.5 * m.dHH;
  double h = sqrt(m.dOH * m.dOH - S.rc * S.rc);
  S.ra = 2.0 * m.mH * h / (m.mO + 2.0 * m.mH);
  S.rb = h - S.ra;
  return S;
}

// The count of inner units that the gated pruning's blocks claim from (the
// deterministic mode keeps the ordered scan: none).
static int32_t *md_unit_counter(mdrtMd &m) {
  NbCtx &c = *m.nb;
  return (c.deterministic || !c.sizes_in) ? nullptr : c.sizes_in + NB_SIZE_UNITS;
}

// The pruning of a step when the update before it asked for it (flag[1],
// on the device): one launch (two in the deterministic mode) that does
// nothing otherwise, no conditional node.
static void md_prune_step(mdrtMd &m, const double *x, const double box[3], cudaStream_t s) {
  NbCtx &c = *m.nb;
  if (c.inner_reach > 0.0)
    nb_prune_gated(c, box, m.flag + 1, x, m.x_prune, m.thermo + 5, md_unit_counter(m), s);
}

// One step on `s` from the frames xq of the current positions x.
static void md_step_body(mdrtMd &m, double *x, double *v, const double box[3], double dt, cudaStream_t s,
                         cudaGraphConditionalHandle h_any, int use_graph, int *flag, int k, int check_build,
                         int window) {
  NbCtx &c = *m.nb;
  bool pme = c.pme.on && c.beta > 0.0;
  bool fused = pme && m.qgrid != nullptr;
  if (pme) {
    cudaEventRecord(m.ev_fork, s);
    cudaStreamWaitEvent(m.side, m.ev_fork, 0);
    if (fused)
      nb_pme_md_chain(c, box, m.qgrid, m.qfixed, m.spec, m.phi, m.influence, flag + 3, m.side);
    else
      nb_pme_run(c, box, false, false, m.side);
  }
  // the pruning that the last update asked for, beside the PME chain (it
  // needs only the frames, and the pair kernel after it needs its lists)
  if (nb_fused_prune(c) && md_unit_counter(m)) {
    // a pruning step prunes and computes its pairs in one kernel (MDIR
    // D284); the pair kernel after it then returns at once
    nb_prune_pairs_run(c, box, m.flag + 1, x, m.x_prune, m.thermo + 5, md_unit_counter(m), s, flag + 3);
    nb_pairs_run(c, box, false, s, flag + 3, m.flag + 1, m.n_excl_other == 0);
  } else {
    md_prune_step(m, x, box, s);
    nb_pairs_run(c, box, false, s, flag + 3, nullptr, m.n_excl_other == 0);
  }
  if (m.n_excl_other > 0) nb_excluded_list_run(c, box, m.excl_other, m.n_excl_other, s);
  if (pme) {
    cudaEventRecord(m.ev_join, m.side);
    cudaStreamWaitEvent(s, m.ev_join, 0);
  }
  UpdateParams U;
  U.noise = m.noise;
  U.k = k;
  U.S = settle_params(m);
  U.dt = dt;
  for (int k = 0; k < 3; ++k) U.L[k] = box[k];
  U.beta = c.beta;
  U.coulomb = c.coulomb;
  U.two_beta_sqrtpi = 2.0 * c.beta / sqrt(M_PI);
  U.water_excl = (m.water_excl && c.beta > 0.0) ? 1 : 0;
  U.fixed = c.deterministic ? 1 : 0;
  U.tau = m.tau;
  U.temperature = m.temperature;
  U.ndof = (double)m.ndof;
  double half = 0.5 * (c.reach - c.cutoff);
  U.build_half2 = half * half;
  double half_in = 0.5 * (c.inner_reach - c.cutoff);
  U.prune_half2 = c.inner_reach > 0.0 ? half_in * half_in : 0.0;
  U.h_any = h_any;
  U.use_graph = use_graph;
  U.flag = flag;
  U.check_build = check_build;
  U.lookahead = m.lookahead;
  U.status = c.status;
  U.peak = m.peak;
  U.pme_fused = fused ? 1 : 0;
  U.G.K0 = c.pme.K[0];
  U.G.K1 = c.pme.K[1];
  U.G.K2 = c.pme.K[2];
  U.G.invL0 = (float)(1.0 / box[0]);
  U.G.invL1 = (float)(1.0 / box[1]);
  U.G.invL2 = (float)(1.0 / box[2]);
  U.phi = m.phi;
  U.host_halt = use_graph ? m.d_halt : nullptr;
  U.unit_counter = c.inner_reach > 0.0 ? md_unit_counter(m) : nullptr;
  nb_launch_chained(md_update, dim3(m.ke_blocks), dim3(MD_UPDATE_THREADS), 0, s, m.nwaters, m.nfree, m.waters,
                    m.free_atoms, U, m.inv_mass, m.mass, c.q, m.wplace, m.fplace, c.shift, c.acc, c.acc_fixed,
                    (pme && !fused) ? (const float4 *)c.pme.pme_force : nullptr, c.xq,
                    c.deterministic ? c.xq_lo : nullptr, x, v, m.force, m.x_ref,
                    m.x_prune, m.thermo, m.ke_part, m.blk_max, m.done_blocks);
}

// A pruning at x on `s` (frames current): the inner lists and their units.
static void md_prune_body(mdrtMd &m, const double *x, const double box[3], cudaStream_t s) {
  NbCtx &c = *m.nb;
  nb_prune_run(c, box, s);
  md_after_prune<<<blocks_for(3 * m.n, 256), 256, 0, s>>>(3 * m.n, x, m.x_prune, m.thermo);
}


// The pruning that the last step asked for, at the end of a run, so that
// the lists in force are valid at the positions the run leaves; no step
// after it prunes again.
static void md_flush_prune(mdrtMd &m, const double *x, const double box[3], cudaStream_t s) {
  md_prune_step(m, x, box, s);
  cudaMemsetAsync(m.flag + 1, 0, sizeof(int), s);
}

// The places by slot after a build (md_places).
static void md_refresh_places(mdrtMd &m, cudaStream_t s) {
  int64_t total = 3 * m.nwaters + m.nfree;
  if (total > 0)
    md_places<<<blocks_for(total, 256), 256, 0, s>>>(3 * m.nwaters, m.nfree, m.waters, m.free_atoms,
                                                    m.nb->place_of, m.wplace, m.fplace);
}

// A build at x on `s` without a host wait (the body of the conditional node).
static void md_rebuild_body(mdrtMd &m, const double *x, const double box[3], cudaStream_t s) {
  NbCtx &c = *m.nb;
  nb_build_launch_public(c, x, box, s);
  nb_gather_frames(c, x, box, s);
  md_refresh_places(m, s);
  md_after_build<<<blocks_for(3 * m.n, 256), 256, 0, s>>>(3 * m.n, x, m.x_ref, m.thermo, c.sizes, c.status,
                                                          m.peak);
}

static void md_drop_graph(mdrtMd *m) {
  if (m->exec) cudaGraphExecDestroy(m->exec);
  if (m->graph) cudaGraphDestroy(m->graph);
  m->exec = nullptr;
  m->graph = nullptr;
}

// The integrator's PME buffers when the update gathers (order 4 with a
// reciprocal sum), sized for the context's grid; none otherwise.
static int md_pme_buffers(mdrtMd *m) {
  NbCtx &c = *m->nb;
  bool want = c.pme.on && c.beta > 0.0 && c.pme.order == 4;
  int64_t pts = want ? (int64_t)c.pme.K[0] * c.pme.K[1] * c.pme.K[2] : 0;
  if (pts == m->pme_points) return 0;
  for (void **p : {(void **)&m->qgrid, (void **)&m->phi, (void **)&m->qfixed, (void **)&m->spec,
                   (void **)&m->influence}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  m->pme_points = 0;
  for (double &k : m->influence_key) k = 0.0;
  if (!want) return 0;
  int64_t half = (int64_t)c.pme.K[0] * c.pme.K[1] * (c.pme.K[2] / 2 + 1);
  if (cudaMalloc(&m->qgrid, sizeof(float) * pts) != cudaSuccess ||
      cudaMalloc(&m->phi, sizeof(float) * pts) != cudaSuccess ||
      cudaMalloc(&m->qfixed, sizeof(unsigned long long) * pts) != cudaSuccess ||
      cudaMalloc(&m->spec, sizeof(float2) * half) != cudaSuccess ||
      cudaMalloc(&m->influence, sizeof(float) * half) != cudaSuccess)
    return -1;
  // the grids start empty; each chain empties the grid it spread (the
  // forward plane kernel of the own transforms; with cuFFT the conversion
  // of the fixed-point grid or the spectrum scaling)
  if (cudaMemset(m->qfixed, 0, sizeof(unsigned long long) * pts) != cudaSuccess ||
      cudaMemset(m->qgrid, 0, sizeof(float) * pts) != cudaSuccess)
    return -1;
  m->pme_points = pts;
  return 0;
}

// The influence table for the MD step's PME chain, made again when the
// cell, the Ewald parameter, the Coulomb factor or the grid differ from
// those it was made for.
static int md_influence(mdrtMd *m, const double box[3], cudaStream_t s) {
  if (!m->influence) return 0;
  const NbCtx &c = *m->nb;
  double key[7] = {box[0], box[1], box[2], c.beta, c.coulomb, (double)c.pme.K[0],
                   (double)c.pme.K[1] * 65536.0 + (double)c.pme.K[2]};
  bool same = true;
  for (int k = 0; k < 7; ++k) same = same && key[k] == m->influence_key[k];
  if (same) return 0;
  if (nb_pme_influence(*m->nb, box, m->influence, s)) return -1;
  for (int k = 0; k < 7; ++k) m->influence_key[k] = key[k];
  return 0;
}

static void md_free(mdrtMd *m) {
  if (!m) return;
  md_drop_graph(m);
  if (m->ev_fork) cudaEventDestroy(m->ev_fork);
  if (m->ev_join) cudaEventDestroy(m->ev_join);
  for (cudaEvent_t e : m->ev_run)
    if (e) cudaEventDestroy(e);
  if (m->h_halt) cudaFreeHost(m->h_halt);
  if (m->side) cudaStreamDestroy(m->side);
  for (void *p : {(void *)m->inv_mass, (void *)m->mass, (void *)m->waters, (void *)m->free_atoms,
                  (void *)m->excl_other, (void *)m->force, (void *)m->x_ref, (void *)m->x_prune,
                  (void *)m->ke_part, (void *)m->done_blocks, (void *)m->blk_max, (void *)m->drift,
                  (void *)m->wplace, (void *)m->fplace, (void *)m->thermo, (void *)m->flag,
                  (void *)m->noise, (void *)m->x_ck, (void *)m->v_ck, (void *)m->thermo_ck, (void *)m->peak,
                  (void *)m->xref_ck, (void *)m->xprune_ck, (void *)m->qgrid, (void *)m->phi, (void *)m->qfixed,
                  (void *)m->spec, (void *)m->influence})
    if (p) cudaFree(p);
  if (m->h_peak) cudaFreeHost(m->h_peak);
  if (m->h_steps) cudaFreeHost(m->h_steps);
  delete m;
}

extern "C" {

int32_t mdrtMdCreate(mdrtMd **out, mdrtNb *nb, const double *masses, int64_t nwaters, const int32_t *waters,
                     double d_oh, double d_hh) {
  if (!out || !nb || !masses || nwaters < 0 || (nwaters > 0 && !waters)) return MDRT_NB_INVALID_ARGUMENT;
  NbCtx &c = nb->c;
  cudaSetDevice(c.device);
  mdrtMd *m = new mdrtMd();
  m->nb = &c;
  m->handle = nb;
  m->device = c.device;
  m->n = c.n;
  m->nwaters = nwaters;
  m->dOH = d_oh;
  m->dHH = d_hh;
  std::vector<int64_t> water_of(c.n, -1);
  for (int64_t w = 0; w < nwaters; ++w)
    for (int k = 0; k < 3; ++k) {
      int32_t a = waters[3 * w + k];
      if (a < 0 || a >= c.n || water_of[a] >= 0) {
        md_free(m);
        return MDRT_NB_INVALID_ARGUMENT;
      }
      water_of[a] = w;
    }
  if (nwaters > 0) {
    m->mO = masses[waters[0]];
    m->mH = masses[waters[1]];
    for (int64_t w = 0; w < nwaters; ++w)
      if (masses[waters[3 * w]] != m->mO || masses[waters[3 * w + 1]] != m->mH ||
          masses[waters[3 * w + 2]] != m->mH) {
        md_free(m);
        return MDRT_NB_UNSUPPORTED;  // one water model per system
      }
  }
  // Excluded pairs: those inside one water go to the update kernel, if every
  // water has all three; the others keep the excluded-pair kernel.
  std::vector<int32_t> pairs(2 * c.n_excl_pairs);
  if (c.n_excl_pairs > 0)
    cudaMemcpy(pairs.data(), c.excl_pairs, sizeof(int32_t) * pairs.size(), cudaMemcpyDeviceToHost);
  std::vector<int> per_water(nwaters, 0);
  std::vector<int32_t> other;
  for (int64_t k = 0; k < c.n_excl_pairs; ++k) {
    int32_t i = pairs[2 * k], j = pairs[2 * k + 1];
    if (water_of[i] >= 0 && water_of[i] == water_of[j])
      per_water[water_of[i]]++;
    else {
      other.push_back(i);
      other.push_back(j);
    }
  }
  bool all = nwaters > 0;
  for (int64_t w = 0; w < nwaters; ++w) all = all && per_water[w] == 3;
  if (!all) {  // keep every pair in the kernel
    other = pairs;
  }
  m->water_excl = all;
  m->n_excl_other = (int64_t)other.size() / 2;
  std::vector<int32_t> fr;
  for (int64_t i = 0; i < c.n; ++i)
    if (water_of[i] < 0) fr.push_back((int32_t)i);
  m->nfree = (int64_t)fr.size();
  std::vector<double> inv(c.n);
  for (int64_t i = 0; i < c.n; ++i) {
    if (!(masses[i] > 0)) {
      md_free(m);
      return MDRT_NB_INVALID_ARGUMENT;
    }
    inv[i] = 1.0 / masses[i];
  }
  m->ndof = 3 * c.n - 3 * nwaters - 3;
  // blocks of waters (10 a warp), then blocks of free atoms (one a thread)
  m->ke_blocks = (int)((nwaters + MD_UPDATE_THREADS / 32 * 10 - 1) / (MD_UPDATE_THREADS / 32 * 10) +
                       (m->nfree + MD_UPDATE_THREADS - 1) / MD_UPDATE_THREADS);
  if (m->ke_blocks < 1) m->ke_blocks = 1;
  int lo = 0, hi = 0;
  cudaDeviceGetStreamPriorityRange(&lo, &hi);
  bool ok = cudaMalloc(&m->inv_mass, sizeof(double) * c.n) == cudaSuccess &&
            cudaMalloc(&m->mass, sizeof(double) * c.n) == cudaSuccess &&
            cudaMalloc(&m->waters, sizeof(int32_t) * std::max<int64_t>(3 * nwaters, 1)) == cudaSuccess &&
            cudaMalloc(&m->free_atoms, sizeof(int32_t) * std::max<int64_t>(m->nfree, 1)) == cudaSuccess &&
            cudaMalloc(&m->excl_other, sizeof(int32_t) * std::max<size_t>(other.size(), 2)) == cudaSuccess &&
            cudaMalloc(&m->force, sizeof(double) * 3 * c.n) == cudaSuccess &&
            cudaMalloc(&m->x_ref, sizeof(double) * 3 * c.n) == cudaSuccess &&
            cudaMalloc(&m->x_prune, sizeof(double) * 3 * c.n) == cudaSuccess &&
            cudaMalloc(&m->ke_part, sizeof(double) * m->ke_blocks) == cudaSuccess &&
            cudaMalloc(&m->done_blocks, sizeof(unsigned int)) == cudaSuccess &&
            cudaMalloc(&m->blk_max, sizeof(float2) * m->ke_blocks) == cudaSuccess &&
            cudaMalloc(&m->drift, sizeof(unsigned int) * 2) == cudaSuccess &&
            cudaMalloc(&m->wplace, sizeof(int32_t) * std::max<int64_t>(3 * nwaters, 1)) == cudaSuccess &&
            cudaMalloc(&m->fplace, sizeof(int32_t) * std::max<int64_t>(m->nfree, 1)) == cudaSuccess &&
            cudaMalloc(&m->thermo, sizeof(double) * 8) == cudaSuccess &&
            cudaMalloc(&m->noise, sizeof(double) * 2 * MD_MAX_UNROLL) == cudaSuccess &&
            cudaMalloc(&m->flag, sizeof(int) * 4) == cudaSuccess &&
            cudaMalloc(&m->x_ck, sizeof(double) * 3 * c.n) == cudaSuccess &&
            cudaMalloc(&m->v_ck, sizeof(double) * 3 * c.n) == cudaSuccess &&
            cudaMalloc(&m->thermo_ck, sizeof(double) * 8) == cudaSuccess &&
            cudaMalloc(&m->xref_ck, sizeof(double) * 3 * c.n) == cudaSuccess &&
            cudaMalloc(&m->xprune_ck, sizeof(double) * 3 * c.n) == cudaSuccess &&
            cudaMalloc(&m->peak, sizeof(int32_t) * 4) == cudaSuccess &&
            cudaMallocHost(&m->h_peak, sizeof(int32_t) * 4) == cudaSuccess &&
            cudaMallocHost(&m->h_steps, sizeof(double) * 2) == cudaSuccess &&
            cudaStreamCreateWithPriority(&m->side, cudaStreamNonBlocking, hi) == cudaSuccess &&
            cudaEventCreateWithFlags(&m->ev_fork, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&m->ev_join, cudaEventDisableTiming) == cudaSuccess &&
            cudaHostAlloc(&m->h_halt, sizeof(int), cudaHostAllocMapped) == cudaSuccess &&
            cudaHostGetDevicePointer(&m->d_halt, m->h_halt, 0) == cudaSuccess;
  for (int k = 0; ok && k <= MD_IN_FLIGHT; ++k)
    ok = cudaEventCreateWithFlags(&m->ev_run[k], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    md_free(m);
    return MDRT_NB_CUDA_ERROR;
  }
  cudaMemcpy(m->inv_mass, inv.data(), sizeof(double) * c.n, cudaMemcpyHostToDevice);
  cudaMemcpy(m->mass, masses, sizeof(double) * c.n, cudaMemcpyHostToDevice);
  if (nwaters > 0) cudaMemcpy(m->waters, waters, sizeof(int32_t) * 3 * nwaters, cudaMemcpyHostToDevice);
  if (m->nfree > 0) cudaMemcpy(m->free_atoms, fr.data(), sizeof(int32_t) * m->nfree, cudaMemcpyHostToDevice);
  if (!other.empty())
    cudaMemcpy(m->excl_other, other.data(), sizeof(int32_t) * other.size(), cudaMemcpyHostToDevice);
  double th[8] = {1.0, 0, 0, 0, 0, 0, 0, 0};
  cudaMemcpy(m->thermo, th, sizeof(th), cudaMemcpyHostToDevice);
  cudaMemset(m->done_blocks, 0, sizeof(unsigned int));
  cudaMemset(m->peak, 0, sizeof(int32_t) * 4);
  cudaMemset(m->flag, 0, sizeof(int) * 4);
  cudaMemset(m->force, 0, sizeof(double) * 3 * c.n);
  *out = m;
  return MDRT_NB_OK;
}

int32_t mdrtMdDestroy(mdrtMd *m) {
  if (m) {
    cudaSetDevice(m->device);
    md_free(m);
  }
  return MDRT_NB_OK;
}

int32_t mdrtMdSetLookahead(mdrtMd *m, double factor) {
  if (!m || !(factor >= 0.0) || !(factor <= 100.0)) return MDRT_NB_INVALID_ARGUMENT;
  m->lookahead = factor;
  md_drop_graph(m);  // parameters are baked into the graph
  return MDRT_NB_OK;
}

int32_t mdrtMdSetThermostat(mdrtMd *m, double temperature, double tau, uint64_t seed) {
  if (!m || !(temperature >= 0)) return MDRT_NB_INVALID_ARGUMENT;
  m->temperature = temperature;
  m->tau = tau;
  m->seed = seed;
  md_drop_graph(m);  // parameters are baked into the graph
  // the scaling the last step computed for the next one belongs to the old
  // thermostat: the next step starts unscaled
  double one = 1.0;
  cudaSetDevice(m->device);
  if (cudaMemcpy(m->thermo, &one, sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) return MDRT_NB_CUDA_ERROR;
  return MDRT_NB_OK;
}

// A build at x that also writes the frames and resets the reference
// positions of the test of validity.
int32_t mdrtMdBuild(mdrtMd *m, const double *x, const double box[3], void *stream) {
  if (!m || !x || !box) return MDRT_NB_INVALID_ARGUMENT;
  int32_t sizes[NB_SIZE_COUNT];
  int32_t s = mdrtNbBuild(m->handle, x, m->n, box, 0.0, stream, sizes);
  if (s) return s;
  cudaStream_t st = (cudaStream_t)stream;
  NbCtx &c = *m->nb;
  if (sizes[NB_SIZE_LONGEST] > NB_GROW_AHEAD * c.list_cap && nb_grow_lists_keep(c, sizes[NB_SIZE_LONGEST], st))
    return MDRT_NB_CUDA_ERROR;
  nb_gather_frames(c, x, box, st);
  md_refresh_places(*m, st);
  if (md_pme_buffers(m)) return MDRT_NB_CUDA_ERROR;
  md_after_build<<<blocks_for(3 * m->n, 256), 256, 0, st>>>(3 * m->n, x, m->x_ref, m->thermo, c.sizes, c.status,
                                                            m->peak);
  if (c.inner_reach > 0.0) {
    md_prune_body(*m, x, box, st);
    c.inner_valid = true;
    c.prunes++;
  }
  cudaMemsetAsync(m->flag + 1, 0, sizeof(int), st);  // pruned here: none due
  return cudaGetLastError() == cudaSuccess ? MDRT_NB_OK : MDRT_NB_CUDA_ERROR;
}

int32_t mdrtMdRefresh(mdrtMd *m, const double *x, const double box[3], void *stream, int32_t *built) {
  if (!m || !x || !box) return MDRT_NB_INVALID_ARGUMENT;
  NbCtx &c = *m->nb;
  cudaStream_t st = (cudaStream_t)stream;
  bool dual = c.inner_reach > 0.0;
  bool same_cell = c.built && box[0] == c.box_built[0] && box[1] == c.box_built[1] && box[2] == c.box_built[2];
  if (same_cell && (!dual || c.inner_valid)) {
    MD_CK(cudaSetDevice(m->device));
    MD_CK(cudaMemsetAsync(m->drift, 0, sizeof(unsigned int) * 2, st));
    md_drift<<<blocks_for(m->n, 256), 256, 0, st>>>(m->n, x, m->x_ref, dual ? m->x_prune : nullptr, m->drift);
    unsigned int h[2] = {0u, 0u};
    MD_CK(cudaMemcpyAsync(h, m->drift, sizeof(h), cudaMemcpyDeviceToHost, st));
    MD_CK(cudaStreamSynchronize(st));
    float d2, p2;
    std::memcpy(&d2, &h[0], sizeof(float));
    std::memcpy(&p2, &h[1], sizeof(float));
    double half = 0.5 * (c.reach - c.cutoff), half_in = 0.5 * (c.inner_reach - c.cutoff);
    // the test of every step of the update: the lists serve x while the
    // largest drift from their build stays within half the skin
    if ((double)d2 <= half * half) {
      nb_gather_frames(c, x, box, st);
      // the pruning that the update would ask for after this drift
      int prune = (dual && (double)p2 > half_in * half_in) ? 1 : 0;
      int flags[4] = {0, prune, 0, 0};
      MD_CK(cudaMemcpyAsync(m->flag, flags, sizeof(flags), cudaMemcpyHostToDevice, st));
      int32_t *counter = md_unit_counter(*m);
      if (prune && counter) MD_CK(cudaMemsetAsync(counter, 0, sizeof(int32_t), st));
      MD_CK(cudaStreamSynchronize(st));
      if (built) *built = 0;
      return MDRT_NB_OK;
    }
  }
  if (built) *built = 1;
  return mdrtMdBuild(m, x, box, stream);
}

}  // extern "C"

// Captures one conditional node (IF) after the current capture point of
// `cap` and the launches of `fill` on `body` into its body graph.
template <typename F>
static cudaError_t md_capture_if(cudaStream_t cap, cudaStream_t body, cudaGraphConditionalHandle h, F &&fill) {
  cudaStreamCaptureStatus status;
  cudaGraph_t g;
  const cudaGraphNode_t *deps = nullptr;
  size_t ndeps = 0;
  cudaError_t e = cudaStreamGetCaptureInfo(cap, &status, nullptr, &g, &deps, &ndeps);
  if (e != cudaSuccess) return e;
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeIf;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  e = cudaGraphAddNode(&node, g, deps, ndeps, &cp);
  if (e != cudaSuccess) return e;
  e = cudaStreamUpdateCaptureDependencies(cap, &node, 1, cudaStreamSetCaptureDependencies);
  if (e != cudaSuccess) return e;
  e = cudaStreamBeginCaptureToGraph(body, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                    cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return e;
  fill(body);
  return cudaStreamEndCapture(body, nullptr);
}

// Steps between the rebuild decisions of the step-by-step path by default
// (the graph path decides at the end of each graph, every `unroll` steps).
#define MD_WINDOW 10

// Step by step, the host reading the flags after each step: a rebuild
// decided ahead at the end of each window of MD_WINDOW steps, or forced by
// a drift past half the skin; the pruning is decided on the device.
static int32_t md_run_steps(mdrtMd *m, double *x, double *v, const double box[3], double dt, int64_t steps,
                            int window, void *stream) {
  cudaStream_t st = (cudaStream_t)stream;
  int h_flag[3] = {0, 0, 0};
  int64_t kw = 0;  // the step in the window; a forced rebuild starts a new window, as in the graphs
  for (int64_t k = 0; k < steps; ++k) {
    md_noise<<<1, 32, 0, st>>>(m->thermo, m->noise, 1, (double)m->ndof, m->seed);
    int check = (kw + 1) % window == 0 ? 1 : 0;
    md_step_body(*m, x, v, box, dt, st, 0, 0, m->flag, 0, check, window);
    cudaMemcpyAsync(h_flag, m->flag, sizeof(h_flag), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return MDRT_NB_CUDA_ERROR;
    ++kw;
    if (h_flag[0] || h_flag[2]) {
      int32_t s = mdrtMdBuild(m, x, box, stream);
      if (s) return s;
      if (h_flag[2]) {
        kw = 0;
        m->redone++;
      }
    }
  }
  md_flush_prune(*m, x, box, st);
  return cudaGetLastError() == cudaSuccess ? MDRT_NB_OK : MDRT_NB_CUDA_ERROR;
}

// Back to the checkpoint of a run: positions, velocities, the lists built
// and pruned where those in force were (no host build of its own: the
// capacities are the caller's), the frames, the thermostat state.
static int32_t md_restore(mdrtMd *m, double *x, double *v, const double box[3], bool dual, void *stream) {
  NbCtx &c = *m->nb;
  cudaStream_t st = (cudaStream_t)stream;
  size_t bytes = sizeof(double) * 3 * m->n;
  if (cudaMemcpyAsync(x, m->x_ck, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(v, m->v_ck, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return MDRT_NB_CUDA_ERROR;
  int32_t s = mdrtNbBuild(m->handle, m->xref_ck, m->n, box, 0.0, stream, nullptr);
  if (s) return s;
  md_refresh_places(*m, st);
  if (cudaMemcpyAsync(m->x_ref, m->xref_ck, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return MDRT_NB_CUDA_ERROR;
  if (dual) {
    nb_gather_frames(c, m->xprune_ck, box, st);
    md_prune_body(*m, m->xprune_ck, box, st);
    c.inner_valid = true;
  }
  cudaMemsetAsync(m->flag + 1, 0, sizeof(int), st);  // a run starts with no pruning due
  nb_gather_frames(c, x, box, st);
  // the counters of the checkpoint: the build and pruning above redo ones it had
  if (cudaMemcpyAsync(m->thermo, m->thermo_ck, sizeof(double) * 8, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return MDRT_NB_CUDA_ERROR;
  return MDRT_NB_OK;
}

// The graph of `unroll` steps (gated prunings, one conditional rebuild at
// the end), captured again when its arguments or the capacities changed.
static int32_t md_prepare_graph(mdrtMd *m, double *x, double *v, const double box[3], double dt, int32_t unroll) {
  NbCtx &c = *m->nb;
  int64_t key = c.groups_cap * 1000003 + c.list_cap * 7 + c.units_cap + (int64_t)(c.inner_reach * 1e9) +
                (c.inner_valid ? 1 : 0) + (c.deterministic ? 2 : 0) + ((int64_t)c.pair_blocks_per_sm << 40) +
                ((int64_t)c.pair_sms << 44) + (int64_t)(uintptr_t)m->qgrid + ((int64_t)nb_fused_prune(c) << 56) +
                ((int64_t)c.staging_depth << 58) + ((int64_t)nb_fft_own(c) << 61) +
                ((int64_t)nb_pme_tiled(c) << 62);
  bool stale = !m->exec || m->gx != x || m->gv != v || m->gdt != dt || m->gunroll != unroll ||
               m->gbox[0] != box[0] || m->gbox[1] != box[1] || m->gbox[2] != box[2] || m->gcap_key != key;
  if (stale) {
    md_drop_graph(m);
    // A window of `unroll` steps: each step prunes when its update asks
    // (gated launches, no conditional node), and the last step decides the
    // rebuild for the window ahead in the graph's one conditional node (an
    // untaken conditional node costs about as much as a short kernel chain,
    // so there is one per window, not one per step).
    cudaStream_t cap, body;
    cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
    cudaStreamCreateWithFlags(&body, cudaStreamNonBlocking);
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    m->handles.assign(1, 0);
    if (e == cudaSuccess)
      md_noise<<<(unroll + 31) / 32, 32, 0, cap>>>(m->thermo, m->noise, unroll, (double)m->ndof, m->seed);
    for (int k = 0; k < unroll && e == cudaSuccess; ++k) {
      bool last = k == unroll - 1;
      if (last) {
        cudaStreamCaptureStatus status;
        cudaGraph_t g;
        e = cudaStreamGetCaptureInfo(cap, &status, nullptr, &g, nullptr, nullptr);
        if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&m->handles[0], g, 0, cudaGraphCondAssignDefault);
        if (e != cudaSuccess) break;
      }
      md_step_body(*m, x, v, box, dt, cap, m->handles[0], 1, m->flag, k, last ? 1 : 0, unroll);
      if (last) e = md_capture_if(cap, body, m->handles[0], [&](cudaStream_t b) { md_rebuild_body(*m, x, box, b); });
    }
    cudaGraph_t graph = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(cap, &graph);
    cudaStreamDestroy(body);
    cudaStreamDestroy(cap);
    if (e != cudaSuccess || e2 != cudaSuccess) {
      fprintf(stderr, "mdrt_nb: step graph capture: %s / %s\n", cudaGetErrorString(e), cudaGetErrorString(e2));
      if (graph) cudaGraphDestroy(graph);
      cudaGetLastError();
      return MDRT_NB_CUDA_ERROR;
    }
    e = cudaGraphInstantiate(&m->exec, graph, cudaGraphInstantiateFlagUseNodePriority);
    if (e != cudaSuccess) {
      fprintf(stderr, "mdrt_nb: step graph instantiate: %s\n", cudaGetErrorString(e));
      cudaGraphDestroy(graph);
      return MDRT_NB_CUDA_ERROR;
    }
    m->graph = graph;
    m->gx = x;
    m->gv = v;
    m->gdt = dt;
    m->gunroll = unroll;
    m->gcap_key = key;
    for (int k = 0; k < 3; ++k) m->gbox[k] = box[k];
  }
  return MDRT_NB_OK;
}

// v += sign dt/2 F/m: the half kick of velocity Verlet at a run's end
// (sign +1) or, backwards, at its start (sign -1).
__global__ void md_half_kick(int64_t n3, const double *__restrict__ f, const double *__restrict__ inv_mass,
                             double half_dt, double *__restrict__ v) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n3) v[i] += half_dt * inv_mass[i / 3] * f[i];
}

// The forces of the term at x (with the lists in force) and the half kick.
static int32_t md_verlet_kick(mdrtMd *m, const double *x, double *v, const double box[3], double half_dt,
                              cudaStream_t st) {
  int32_t s = mdrtNbForce(m->handle, x, box, 0u, m->force, st);
  if (s) return s;
  md_half_kick<<<blocks_for(3 * m->n, 256), 256, 0, st>>>(3 * m->n, m->force, m->inv_mass, half_dt, v);
  return cudaGetLastError() == cudaSuccess ? MDRT_NB_OK : MDRT_NB_CUDA_ERROR;
}

static int32_t md_run_leapfrog(mdrtMd *m, double *x, double *v, const double box[3], double dt, int64_t steps,
                               int32_t unroll, void *stream);

extern "C" {

int32_t mdrtMdSetIntegrator(mdrtMd *m, int32_t method) {
  if (!m || (method != MDRT_MD_LEAP_FROG && method != MDRT_MD_VELOCITY_VERLET)) return MDRT_NB_INVALID_ARGUMENT;
  // velocities on the step need the velocity constraints of rigid waters
  // (RATTLE), which the step does not apply
  if (method == MDRT_MD_VELOCITY_VERLET && m->nwaters > 0) return MDRT_NB_UNSUPPORTED;
  m->verlet = method == MDRT_MD_VELOCITY_VERLET;
  return MDRT_NB_OK;
}

// Velocity Verlet and leap-frog give the same positions; they differ in
// when the velocities are: on the step (v_n) or half a step behind.  With
// velocity Verlet the run takes v_0, turns it into v_{-1/2} = v_0 - F_0
// dt/(2m), runs the leap-frog steps, and turns v_{N-1/2} into v_N =
// v_{N-1/2} + F_N dt/(2m), with the forces at the run's first and last
// positions (two evaluations of the term a run).
int32_t mdrtMdRun(mdrtMd *m, double *x, double *v, const double box[3], double dt, int64_t steps,
                  int32_t unroll, void *stream) {
  if (!m || !x || !v || !box || !(dt > 0) || steps < 0 || unroll > MD_MAX_UNROLL || unroll < -MD_MAX_UNROLL)
    return MDRT_NB_INVALID_ARGUMENT;
  if (!m->verlet || steps == 0) return md_run_leapfrog(m, x, v, box, dt, steps, unroll, stream);
  NbCtx &c = *m->nb;
  if (!c.built) return MDRT_NB_NOT_BUILT;
  cudaSetDevice(c.device);
  cudaStream_t st = (cudaStream_t)stream;
  int32_t s = md_verlet_kick(m, x, v, box, -0.5 * dt, st);
  if (!s) s = md_run_leapfrog(m, x, v, box, dt, steps, unroll, stream);
  if (!s) s = md_verlet_kick(m, x, v, box, 0.5 * dt, st);
  return s;
}

}  // extern "C"

static int32_t md_run_leapfrog(mdrtMd *m, double *x, double *v, const double box[3], double dt, int64_t steps,
                               int32_t unroll, void *stream) {
  if (!m || !x || !v || !box || !(dt > 0) || steps < 0 || unroll > MD_MAX_UNROLL || unroll < -MD_MAX_UNROLL)
    return MDRT_NB_INVALID_ARGUMENT;
  NbCtx &c = *m->nb;
  if (!c.built) return MDRT_NB_NOT_BUILT;
  for (int k = 0; k < 3; ++k)
    if (box[k] != c.box_built[k]) return MDRT_NB_INVALID_BOX;
  cudaSetDevice(c.device);
  cudaStream_t st = (cudaStream_t)stream;
  if (md_influence(m, box, st)) return MDRT_NB_CUDA_ERROR;
  md_refresh_places(*m, st);  // the term may have been built without the integrator
  if (unroll <= 0) return md_run_steps(m, x, v, box, dt, steps, unroll < 0 ? -unroll : MD_WINDOW, stream);
  // Runs of step graphs.  Each run starts from a checkpoint (positions,
  // velocities, thermostat state, and the positions the lists in force were
  // built and pruned at) and ends in one read of what its steps saw.  A
  // rebuild inside a graph that overflowed a list: back to the checkpoint,
  // the lists grown to the longest count (+25%), built and pruned again
  // where they were (the same lists and schedule, with room), and the run
  // again.  A drift past half the skin between two rebuild decisions (the
  // decision looks ahead, so this is rare): the steps after it did nothing,
  // so the host rebuilds at that step and runs the steps left.  Positions
  // that are not finite end the run.
  size_t bytes = sizeof(double) * 3 * m->n;
  bool dual = c.inner_reach > 0.0 && c.inner_valid;
  int64_t left = steps;
  for (int attempt = 0; left >= unroll;) {
    int64_t launches = left / unroll;
    int32_t s = md_prepare_graph(m, x, v, box, dt, unroll);
    if (s) return s;
    if (cudaMemcpyAsync(m->x_ck, x, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(m->v_ck, v, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(m->xref_ck, m->x_ref, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
        (dual && cudaMemcpyAsync(m->xprune_ck, m->x_prune, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess) ||
        cudaMemcpyAsync(m->thermo_ck, m->thermo, sizeof(double) * 8, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
        cudaMemsetAsync(m->peak, 0, sizeof(int32_t) * 4, st) != cudaSuccess)
      return MDRT_NB_CUDA_ERROR;
    // the previous run ended in a synchronize: nothing writes the word now
    *(volatile int *)m->h_halt = 0;
    for (int64_t k = 0; k < launches; ++k) {
      cudaEvent_t &done = m->ev_run[k % (MD_IN_FLIGHT + 1)];
      if (k > MD_IN_FLIGHT) {
        // the graph launched MD_IN_FLIGHT + 1 launches ago has finished
        // (the ones after it keep the device busy meanwhile)
        if (cudaEventSynchronize(done) != cudaSuccess) return MDRT_NB_CUDA_ERROR;
        if (*(volatile int *)m->h_halt) break;
      }
      if (cudaGraphLaunch(m->exec, st) != cudaSuccess || cudaEventRecord(done, st) != cudaSuccess)
        return MDRT_NB_CUDA_ERROR;
    }
    if (cudaMemcpyAsync(m->h_peak, m->peak, sizeof(int32_t) * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(m->h_steps, m->thermo_ck + 3, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(m->h_steps + 1, m->thermo + 3, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return MDRT_NB_CUDA_ERROR;
    if (m->h_peak[2] > 0) return MDRT_NB_NAN_POSITION;
    if (m->h_peak[1] != 0) {
      if (++attempt > 8) return MDRT_NB_GROW;
      md_clear_status<<<1, 1, 0, st>>>(c.status, NB_STATUS_LIST_OVERFLOW | NB_STATUS_STALE_LIST);
      if (cudaMemsetAsync(m->flag + 3, 0, sizeof(int), st) != cudaSuccess) return MDRT_NB_CUDA_ERROR;
      if (nb_grow_lists(c, m->h_peak[0])) return MDRT_NB_CUDA_ERROR;
      s = md_restore(m, x, v, box, dual, stream);
      if (s) return s;
      m->regrows++;
      continue;
    }
    if (m->h_peak[3] != 0) {
      // stopped at a stale list: rebuild there and go on with the steps left
      int64_t done = (int64_t)(m->h_steps[1] - m->h_steps[0]);
      md_clear_status<<<1, 1, 0, st>>>(c.status, NB_STATUS_STALE_LIST);
      if (cudaMemsetAsync(m->flag + 3, 0, sizeof(int), st) != cudaSuccess) return MDRT_NB_CUDA_ERROR;
      s = mdrtMdBuild(m, x, box, stream);
      if (s) return s;
      m->redone++;
      left -= done;
      continue;
    }
    // lists near their capacity grow ahead, keeping those in force
    if (m->h_peak[0] > NB_GROW_AHEAD * c.list_cap && nb_grow_lists_keep(c, m->h_peak[0], st))
      return MDRT_NB_CUDA_ERROR;
    left -= launches * unroll;
  }
  md_flush_prune(*m, x, box, st);
  if (left > 0) return md_run_steps(m, x, v, box, dt, left, unroll, stream);
  return cudaGetLastError() == cudaSuccess ? MDRT_NB_OK : MDRT_NB_CUDA_ERROR;
}

extern "C" {

// [0] lambda, [1] kinetic energy of the last half step, [2] of the one
// before, [3] steps, [4] builds since create, [5] degrees of freedom.
int32_t mdrtMdThermo(mdrtMd *m, void *stream, double *out) {
  if (!m || !out) return MDRT_NB_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  double h[8];
  if (cudaMemcpyAsync(h, m->thermo, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess) return MDRT_NB_CUDA_ERROR;
  if (cudaStreamSynchronize(st) != cudaSuccess) return MDRT_NB_CUDA_ERROR;
  for (int k = 0; k < 5; ++k) out[k] = h[k];
  out[5] = (double)m->ndof;
  out[6] = h[5];
  out[7] = (double)m->regrows;
  out[8] = (double)m->redone;
  return MDRT_NB_OK;
}

// The forces of the last step (device f64 [n, 3]).
int32_t mdrtMdForces(mdrtMd *m, double **forces) {
  if (!m || !forces) return MDRT_NB_INVALID_ARGUMENT;
  *forces = m->force;
  return MDRT_NB_OK;
}

}  // extern "C"
