// The Lennard-Jones + Ewald real-space pair kernel on sm_100a, the excluded
// pair correction, the frame gather and the force / energy finish.
//
// Replaces MDIR's emitted pair loop (lib/Conversion/MDExecKernels/
// TraversePairs.cpp:85 emitGroupPairKernel; schedule in
// docs/neighbor-groups.md:533-594) and the excluded-pair tuple loop
// (lib/Driver/TermNonbonded.cpp:1615-1671).  Physics as
// TermNonbonded.cpp:378-466 and TermLennardJones.cpp:26-80: for each
// unordered pair in the lists with r^2 < rc^2 (strict), LJ from a table of
// (c6, c12) by type pair and f q_i q_j (erfc(beta r)/r - shift).
//
// Schedule (B200 design): a warp takes a unit of <= 64 entries of one group
// in two rounds of 32.  Each lane keeps its own entry (partner place, mask,
// image) and its partner's position in registers for the whole round; the
// 16 members are read from shared memory, lane l taking member (l + k) mod
// 16 at step k, so the 32 lanes visit 32 different (member, entry) slots
// per step.  The member's force accumulator travels with the member: after
// each step it moves one lane down the half-warp (3 shuffles), and after 16
// steps it is home again.  The partner's force stays in its lane and is
// added once per entry with one float4 atomic (red.global.add.v4.f32), or
// three 64-bit integer atomics in fixed point in the deterministic mode.
// A round whose 32 entries all have at most NB_SPARSE_BITS members (the
// pruned lists put those entries last, by member count) skips the 16 steps:
// each lane visits its own members only, one a step, and the member forces
// are summed from shared memory in lane order after the round.
// Energies and virial go to a per-unit f64 slot, summed later in a fixed
// order, so they are bitwise reproducible in every mode.
#include <cmath>
#include <cstdio>

#include "nb_context.h"
#include "nb_prune.cuh"

#define NB_MAX_TYPES 32

namespace {

struct PairParams {
  float Lx, Ly, Lz;
  float bx, cx, cy;  // tilts of a triclinic cell (0: orthorhombic)
  double Ld[6];      // the cell in f64 (ax, by, cz, bx, cx, cy): the exact image shifts of the split frames
  int update_after;  // the MD step: the update chained after the kernel may start beside it
  float rc2;
  float beta;
  float beta_p;         // p beta, p of the erfc approximation below
  float nb2_log2e;      // -beta^2 log2(e): exp(-beta^2 r^2) = 2^(r^2 nb2_log2e)
  float two_beta_sqrtpi;
  float coulomb;
  float coulomb_shift;  // erfc(beta rc)/rc when the direct sum is shifted, else 0
  float rs2, winv;      // LJ switch 1, in r^2: rs^2 and 1 / (rc^2 - rs^2)
  float rs, winv_r;     // LJ switch 2, in r: rs and 1 / (rc - rs)
  int ntypes;
  int64_t list_cap;
  int64_t units_cap;
};

// The special-function unit's approximations with denormals flushed
// (PTX rsqrt/ex2/rcp .approx.ftz).  The flush touches only arguments or
// results below 2^-126: r^2 that small means two sites at one point, and
// 2^(r^2 nb2_log2e) stays above 2^-40 within any cutoff for which the real
// space sum is accurate (beta r_c <= 5), so no value changes and the
// denormal scaling of the non-ftz forms is dropped.
__device__ __forceinline__ float nb_rsqrt(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float nb_ex2(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float nb_rcp(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// erfc(beta r) from exp(-beta^2 r^2): Abramowitz & Stegun 7.1.26
// (Hastings), |error| <= 1.5e-7, with t = 1 / (1 + p beta r).  `pbr` is
// p beta r; `ex` is exp(-beta^2 r^2), computed once and shared with the force.
__device__ __forceinline__ float nb_erfc_from_exp(float pbr, float ex) {
  const float a1 = 0.254829592f, a2 = -0.284496736f, a3 = 1.421413741f, a4 = -1.453152027f,
              a5 = 1.061405429f;
  float t = nb_rcp(1.0f + pbr);
  float poly = fmaf(fmaf(fmaf(fmaf(a5, t, a4), t, a3), t, a2), t, a1) * t;
  return poly * ex;
}

// One pair at r2 with LJ factors cc = (6 c6, 12 c12) and charge product qq
// (times the Coulomb constant): the force factor fs (the force on the member
// is fs d, d its displacement from the partner) and, with ENERGY, the LJ and
// Coulomb energies.  A pair outside (masked, or beyond r_c) computes on its
// own r^2, finite or not; the caller drops its results.
// SWITCH multiplies the LJ potential by S from rs to rc: 1, the cubic in r^2
// S = (1 - y)^2 (1 + 2y), y = (r^2 - rs^2)/(rc^2 - rs^2) (MDIR's
// SQUARED_DISTANCE_SWITCH modifier, TermLennardJones.cpp:72-95); 2, the
// quintic in r S = 1 - 10t^3 + 15t^4 - 6t^5, t = (r - rs)/(rc - rs) (the
// potential switch of MDIR's md dialect, ExpandTruncation.cpp:19-46).
template <bool ENERGY, int SWITCH>
__device__ __forceinline__ void nb_pair_terms(const PairParams &P, float r2, float2 cc, float qq, float &fs,
                                              float &ulj, float &uc) {
  float rinv = nb_rsqrt(r2);
  float rinv2 = rinv * rinv;
  float s6 = rinv2 * rinv2 * rinv2;
  float a12 = cc.y * s6 * s6, a6 = cc.x * s6;  // 12 c12 / r^12, 6 c6 / r^6
  fs = (a12 - a6) * rinv2;
  ulj = (ENERGY || SWITCH) ? a12 * (1.f / 12.f) - a6 * (1.f / 6.f) : 0.f;
  float rr = r2 * rinv;
  if (SWITCH == 1) {
    float y = fminf(fmaxf((r2 - P.rs2) * P.winv, 0.f), 1.f);
    float S = (1.f - y) * (1.f - y) * (1.f + 2.f * y);
    float dSdr2 = -6.f * y * (1.f - y) * P.winv;
    fs = fs * S - 2.f * ulj * dSdr2;
    ulj *= S;
  } else if (SWITCH == 2) {
    float t = fminf(fmaxf((rr - P.rs) * P.winv_r, 0.f), 1.f);
    float S = fmaf(t * t * t, fmaf(t, fmaf(-6.f, t, 15.f), -10.f), 1.f);
    float dSdr = t * t * fmaf(t, fmaf(-30.f, t, 60.f), -30.f) * P.winv_r;
    fs = fs * S - ulj * dSdr * rinv;  // -(dU/dr S + U dS/dr) / r
    ulj *= S;
  }
  float ex = nb_ex2(r2 * P.nb2_log2e);
  float erfcv = nb_erfc_from_exp(P.beta_p * rr, ex);
  fs = fmaf(qq * fmaf(erfcv, rinv, P.two_beta_sqrtpi * ex), rinv2, fs);
  uc = ENERGY ? qq * (erfcv * rinv - P.coulomb_shift) : 0.f;
}

__device__ __forceinline__ void nb_red_add_v4(float4 *addr, float x, float y, float z) {
  // one vector reduction instead of three (sm_90 and newer)
  atomicAdd(addr, make_float4(x, y, z, 0.f));
}

__device__ __forceinline__ void nb_red_fixed(unsigned long long *addr, float x, float y, float z,
                                             int *status) {
  if (fabsf(x) > 1e9f || fabsf(y) > 1e9f || fabsf(z) > 1e9f) atomicOr(status, NB_STATUS_FIXED_OVERFLOW);
  atomicAdd(addr + 0, (unsigned long long)__float2ll_rn(x * 4294967296.0f));
  atomicAdd(addr + 1, (unsigned long long)__float2ll_rn(y * 4294967296.0f));
  atomicAdd(addr + 2, (unsigned long long)__float2ll_rn(z * 4294967296.0f));
}

// One unit of a list (group g = uo.x, entries 64 uo.y ... 64 uo.y + 63) by
// one warp: the rounds of 32 entries (dense, or sparse for entries of at
// most NB_SPARSE_BITS members), the members' and partners' forces, and with
// ENERGY the unit's energy and virial partials at `unit`.  s_xw, s_fw, s_tw
// and s_bw are the warp's shared arrays (the 16 members twice; the sparse
// round's member forces).  With STAGED the caller has read the unit's two
// rounds of entries ahead (pre0, pre1: the staging depth 2 of the pair
// kernel); else the force forms read them here, in flight with the
// members' loads.
//
// FIXED (the deterministic mode) takes split frames: the f32 frame xq and
// its rounding residual xq_lo ((x + (S - 1/2) L) - xq in f32), the
// partner's image shift exact in f64 and split the same way, so that a
// pair's displacement is (xm - xj) + (xm_lo - xj_lo): no bits lost to the
// size of the cell (a 22 nm box has f32 frames of up to 11 nm).  s_lw is
// the warp's shared array of the members' residuals.
template <bool ENERGY, bool FIXED, int SWITCH, int LJM, bool BATCH, bool STAGED = false>
__device__ __forceinline__ void nb_pair_unit(const PairParams &P, int2 uo, int64_t unit, int2 pre0, int2 pre1,
                                             const float4 *__restrict__ group_L, const int2 *__restrict__ slab,
                                             const int32_t *__restrict__ counts, const float4 *__restrict__ xq,
                                             const float4 *__restrict__ xq_lo, float4 *s_lw,
                                             const int32_t *__restrict__ typ, const float2 *__restrict__ ljf,
                                             const float2 *s_lj, float4 *s_xw, float2 *s_fw, int *s_tw,
                                             float (*s_bw)[NB_SPARSE_BITS][33], float4 *__restrict__ acc,
                                             unsigned long long *__restrict__ accf, double *__restrict__ partials,
                                             int *__restrict__ status) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31, u = lane & 15;
  const int src = (lane & 16) | ((lane + 1) & 15);  // the lane the member accumulators come from
  int g = uo.x;
  int64_t pi = (int64_t)g * NB_GROUP + u;
  // both rounds' entries, in flight with the members' loads (a group's
  // slab holds a whole number of units, so both reads stay in it; the
  // lanes past the list's end drop theirs below); the energy forms read
  // each round's when they come to it
  const int2 *row = slab + (int64_t)g * P.list_cap + (int64_t)uo.y * NB_UNIT;
  if (!ENERGY && !STAGED) {
    pre0 = row[lane];
    pre1 = row[32 + lane];
  }
  __syncwarp();
  {
    float4 xi = xq[pi];
    xi.w *= P.coulomb;
    int ti = typ[pi];
    s_xw[lane] = xi;
    if (FIXED) s_lw[lane] = xq_lo[pi];
    if (LJM == 1) {  // the member's factors times 6 and 12: the force's factors
      float2 f = ljf[ti];
      s_fw[lane] = make_float2(6.f * f.x, 12.f * f.y);
    } else
      s_tw[lane] = ti * P.ntypes;
  }
  __syncwarp();
  int cnt = (int)min((int64_t)counts[g], P.list_cap);
  int e0 = uo.y * NB_UNIT;
  int ne = min(NB_UNIT, cnt - e0);
  float Lx = P.Lx, Ly = P.Ly, Lz = P.Lz;
  if (BATCH) {  // the cell of the group's frame
    float4 Lg = group_L[g];
    Lx = Lg.x;
    Ly = Lg.y;
    Lz = Lg.z;
  }
  float ax = 0.f, ay = 0.f, az = 0.f;  // the accumulator of member (lane + k) mod 16
  float elj = 0.f, ecl = 0.f;
  float vxx = 0.f, vyy = 0.f, vzz = 0.f, vxy = 0.f, vxz = 0.f, vyz = 0.f;
  for (int r = 0; r < 2; ++r) {
    if (r * 32 >= ne) break;
    bool valid = r * 32 + lane < ne;
    int2 en = valid ? ((ENERGY && !STAGED) ? row[r * 32 + lane] : (r == 0 ? pre0 : pre1)) : make_int2(0, 0);
    int q = en.x;
    unsigned mask = valid ? ((unsigned)en.y & 0xffffu) : 0u;
    int code = ((unsigned)en.y >> 16) & NB_IMAGE_BITS;
    int sx, sy, sz;
    nb_decode_image(code, sx, sy, sz);
    float4 xj = xq[q];
    float3 jl = make_float3(0.f, 0.f, 0.f);  // FIXED: the residual of the partner's image
    if (FIXED) {
      // the image x_j + n H in f64 from the split frame, split again
      float4 lo = xq_lo[q];
      double na = sx, nbv = sy, nc = sz;
      double X = (double)xj.x + (double)lo.x + ((na * P.Ld[0] + nbv * P.Ld[3]) + nc * P.Ld[4]);
      double Y = (double)xj.y + (double)lo.y + (nbv * P.Ld[1] + nc * P.Ld[5]);
      double Z = (double)xj.z + (double)lo.z + nc * P.Ld[2];
      xj.x = (float)X;
      xj.y = (float)Y;
      xj.z = (float)Z;
      jl = make_float3((float)(X - (double)xj.x), (float)(Y - (double)xj.y), (float)(Z - (double)xj.z));
    } else {
      NbCell H;
      H.ax = Lx;
      H.by = Ly;
      H.cz = Lz;
      H.bx = P.bx;
      H.cx = P.cx;
      H.cy = P.cy;
      float3 t = nb_lattice_shift(sx, sy, sz, H);
      xj.x += t.x;
      xj.y += t.y;
      xj.z += t.z;
    }
    int tj = typ[q];
    float2 fj = LJM == 1 ? ljf[tj] : make_float2(0.f, 0.f);
    float fjx = 0.f, fjy = 0.f, fjz = 0.f;
    // One pair of this lane's entry with the member at slot m: its force
    // (dropped outside), the partner's share and the energies.
    auto pair = [&](int m, bool masked_in, float &fx, float &fy, float &fz) {
      float4 xm = s_xw[m];
      float dx = xm.x - xj.x, dy = xm.y - xj.y, dz = xm.z - xj.z;
      if (FIXED) {
        float4 ml = s_lw[m];
        dx += ml.x - jl.x;
        dy += ml.y - jl.y;
        dz += ml.z - jl.z;
      }
      float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
      bool inside = masked_in && (r2 < P.rc2);
      float2 cc;  // (6 c6, 12 c12)
      if (LJM == 1) {
        float2 fm = s_fw[m];
        cc = make_float2(fm.x * fj.x, fm.y * fj.y);
      } else {
        cc = s_lj[s_tw[m] + tj];
      }
      float qq = xm.w * xj.w;
      float fs, ulj, uc;
      nb_pair_terms<ENERGY, SWITCH>(P, r2, cc, qq, fs, ulj, uc);
      fs = inside ? fs : 0.f;
      fx = fs * dx;
      fy = fs * dy;
      fz = fs * dz;
      fjx -= fx;
      fjy -= fy;
      fjz -= fz;
      if (ENERGY) {
        elj += inside ? ulj : 0.f;
        ecl += inside ? uc : 0.f;
        vxx = fmaf(dx, fx, vxx);
        vyy = fmaf(dy, fy, vyy);
        vzz = fmaf(dz, fz, vzz);
        vxy = fmaf(dx, fy, vxy);
        vxz = fmaf(dx, fz, vxz);
        vyz = fmaf(dy, fz, vyz);
      }
    };
    if (__all_sync(FULL, __popc(mask) <= NB_SPARSE_BITS)) {
      // A sparse round (the pruned lists put such entries last): each lane
      // visits only its own members, as many as the fullest entry of the
      // round has.  Its i-th member's force goes to s_b[.][i][lane]; then
      // lanes u and u + 16 add member u's forces over the lanes of their
      // half, in lane order.
      int steps = (int)__reduce_max_sync(FULL, (unsigned)__popc(mask));
      unsigned mm = mask;
      // the next member of this lane's entry, or a dropped pair with
      // member 0 once none is left (a lane with fewer members idles so)
      auto visit = [&](int i) {
        bool has = mm != 0u;
        int m = has ? __ffs(mm) - 1 : 0;
        mm &= mm - 1;
        float fx, fy, fz;
        pair(m, has, fx, fy, fz);
        if (has) {
          s_bw[0][i][lane] = fx;
          s_bw[1][i][lane] = fy;
          s_bw[2][i][lane] = fz;
        }
      };
      // two members a step, branch-free, so that their chains interleave
      int i = 0;
      for (; i + 1 < steps; i += 2) {
        visit(i);
        visit(i + 1);
      }
      if (i < steps) visit(i);
      __syncwarp();
      float sx = 0.f, sy = 0.f, sz = 0.f;
      const unsigned below = (1u << u) - 1u;
#pragma unroll 4
      for (int j = 0; j < 16; ++j) {
        int lp = (lane & 16) | j;
        unsigned mk = __shfl_sync(FULL, mask, lp);
        if ((mk >> u) & 1u) {
          int i = __popc(mk & below);
          sx += s_bw[0][i][lp];
          sy += s_bw[1][i][lp];
          sz += s_bw[2][i][lp];
        }
      }
      __syncwarp();  // the next round writes s_b again
      ax += sx;
      ay += sy;
      az += sz;
    } else {
      // bit k of mrot: the pair of this lane's entry with member (lane + k) mod 16
      unsigned mrot = ((mask >> u) | (mask << (16 - u))) & 0xffffu;
#pragma unroll
      for (int k = 0; k < NB_GROUP; ++k) {
        float fx, fy, fz;
        pair(u + k, (mrot & (1u << k)) != 0u, fx, fy, fz);
        ax += fx;
        ay += fy;
        az += fz;
        ax = __shfl_sync(FULL, ax, src);
        ay = __shfl_sync(FULL, ay, src);
        az = __shfl_sync(FULL, az, src);
      }
    }
    if (valid && (fjx != 0.f || fjy != 0.f || fjz != 0.f)) {
      if (FIXED)
        nb_red_fixed(accf + 3 * (int64_t)q, fjx, fjy, fjz, status);
      else
        nb_red_add_v4(acc + q, fjx, fjy, fjz);
    }
  }
  ax += __shfl_xor_sync(FULL, ax, 16);
  ay += __shfl_xor_sync(FULL, ay, 16);
  az += __shfl_xor_sync(FULL, az, 16);
  if (lane < 16 && (ax != 0.f || ay != 0.f || az != 0.f)) {
    if (FIXED)
      nb_red_fixed(accf + 3 * pi, ax, ay, az, status);
    else
      nb_red_add_v4(acc + pi, ax, ay, az);
  }
  if (ENERGY) {
    double v[8] = {elj, ecl, vxx, vyy, vzz, vxy, vxz, vyz};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(FULL, v[k], o);
    }
    if (lane == 0) {
#pragma unroll
      for (int k = 0; k < 8; ++k) partials[(int64_t)unit * 8 + k] = v[k];
    }
  }
}

// LJM selects the Lennard-Jones coefficients: 0, a (c6, c12) table by type
// pair in shared memory; 1, the product of per-type factors (sqrt c6,
// sqrt c12), exact when the table factorizes (one LJ type, or geometric
// mixing), which needs no dependent lookup.  The members live twice in
// shared memory (slots u and u + 16), so that in a dense round lane l reads
// member (l + k) mod 16 at slot l mod 16 + k: an immediate offset in the
// unrolled loop, no index arithmetic.
// DEPTH is the staging depth: 1, a unit's entries are read when it starts
// (the force forms read the next unit's header during a unit, the energy
// forms each round's entries when they come to it); 2, the next unit's
// header and entries are in flight during a unit (four more registers).
// Warps a block of the pair kernel (a persistent grid of
// pair_blocks_per_sm x 8 / NB_PAIR_WARPS blocks an SM).  The MD step of the
// 23,550-atom box measured 54.2-54.3 µs with 8, 54.9-55.2 with 2 and
// 55.9-56.7 with 1, side by side (unlike the adjoint, no other kernel waits
// for the SMs its early warps would free).
#ifndef NB_PAIR_WARPS
#define NB_PAIR_WARPS 8
#endif
template <bool ENERGY, bool FIXED, int SWITCH, int LJM, bool BATCH = false, int DEPTH = 1>
__global__ void __launch_bounds__(NB_PAIR_WARPS * 32, 32 / NB_PAIR_WARPS) nb_pairs(PairParams P, const float4 *__restrict__ group_L,
                                                const int32_t *__restrict__ sizes,
                                                const int2 *__restrict__ units,
                                                const int2 *__restrict__ slab,
                                                const int32_t *__restrict__ counts,
                                                const float4 *__restrict__ xq,
                                                const float4 *__restrict__ xq_lo,
                                                const int32_t *__restrict__ typ,
                                                const float2 *__restrict__ lj, const float2 *__restrict__ ljf,
                                                float4 *__restrict__ acc, unsigned long long *__restrict__ accf,
                                                double *__restrict__ partials, int *__restrict__ status,
                                                const int *halt, const int *skip) {
  // the MD step's update may start its loads, its PME gather and its
  // excluded pairs beside this kernel; it waits for these forces
  if (P.update_after) nb_grid_launch_dependents();
  nb_grid_wait();  // the lists and frames of the kernels before (a chained launch)
  if (halt && *halt) return;  // the MD step stopped at a stale list (its host rebuilds)
  if (skip && *skip) return;  // a pruning step: the pruning kernel computed the pairs
  __shared__ float4 s_x[NB_PAIR_WARPS][2 * NB_GROUP];
  __shared__ float4 s_l[NB_PAIR_WARPS][FIXED ? 2 * NB_GROUP : 1];  // FIXED: the members' frame residuals
  __shared__ float2 s_f[NB_PAIR_WARPS][2 * NB_GROUP];  // LJM 1: member factors
  __shared__ int s_t[NB_PAIR_WARPS][2 * NB_GROUP];     // LJM 0: member row offsets in s_lj
  __shared__ float2 s_lj[LJM == 0 ? NB_MAX_TYPES * NB_MAX_TYPES : 1];
  __shared__ float s_b[NB_PAIR_WARPS][3][NB_SPARSE_BITS][33];  // member forces of a sparse round (33: no bank conflicts)
  if (LJM == 0) {  // (6 c6, 12 c12): the force's factors
    int nt2 = P.ntypes * P.ntypes;
    for (int k = threadIdx.x; k < nt2; k += blockDim.x) {
      float2 c = lj[k];
      s_lj[k] = make_float2(6.f * c.x, 12.f * c.y);
    }
    __syncthreads();
  }
  int warp = threadIdx.x >> 5;
  int nunits = min((int64_t)sizes[NB_SIZE_UNITS], P.units_cap);
  int wstride = gridDim.x * NB_PAIR_WARPS;
  // the next unit's header is in flight during this unit (the energy forms,
  // short of registers, read it when they come to it)
  int unit = blockIdx.x * NB_PAIR_WARPS + warp;
  const int lane = threadIdx.x & 31;
  if (DEPTH == 2) {
    // the unit's entries were read during the unit before
    int2 uo = unit < nunits ? units[unit] : make_int2(0, 0);
    int2 e0 = make_int2(0, 0), e1 = make_int2(0, 0);
    if (unit < nunits) {
      const int2 *row = slab + (int64_t)uo.x * P.list_cap + (int64_t)uo.y * NB_UNIT;
      e0 = row[lane];
      e1 = row[32 + lane];
    }
    for (; unit < nunits; unit += wstride) {
      int2 un = make_int2(0, 0), n0 = make_int2(0, 0), n1 = make_int2(0, 0);
      if (unit + wstride < nunits) {
        un = units[unit + wstride];
        const int2 *row = slab + (int64_t)un.x * P.list_cap + (int64_t)un.y * NB_UNIT;
        n0 = row[lane];
        n1 = row[32 + lane];
      }
      nb_pair_unit<ENERGY, FIXED, SWITCH, LJM, BATCH, true>(P, uo, unit, e0, e1, group_L, slab, counts, xq, xq_lo,
                                                            s_l[warp], typ, ljf, s_lj, s_x[warp], s_f[warp],
                                                            s_t[warp], s_b[warp], acc, accf, partials, status);
      uo = un;
      e0 = n0;
      e1 = n1;
    }
    return;
  }
  int2 uo_next = !ENERGY && unit < nunits ? units[unit] : make_int2(0, 0);
  for (; unit < nunits; unit += wstride) {
    int2 uo = ENERGY ? units[unit] : uo_next;
    if (!ENERGY && unit + wstride < nunits) uo_next = units[unit + wstride];
    nb_pair_unit<ENERGY, FIXED, SWITCH, LJM, BATCH>(P, uo, unit, make_int2(0, 0), make_int2(0, 0), group_L, slab,
                                                    counts, xq, xq_lo, s_l[warp], typ, ljf, s_lj, s_x[warp],
                                                    s_f[warp], s_t[warp], s_b[warp], acc, accf, partials, status);
  }
}

// The pruning step of the dual list with its pairs in one kernel (MDIR
// D284: the loop over pairs that first takes a pruning prunes for it): a
// block of NB_PRUNE_WARPS warps a group prunes the group's outer list at the
// step's frames exactly as the pruning kernel does (nb_prune_group: the same
// inner list, counts and claimed units, and the positions of the pruning),
// then its warps evaluate the units of that fresh inner list at once, while
// other blocks are still pruning.  Forces only, outside the deterministic
// mode (the claimed units come in block order); nothing unless *gate is set
// (the update before asked for a pruning) and the step goes on.
template <int SWITCH, int LJM>
__global__ void __launch_bounds__(NB_PRUNE_WARPS * 32)
    nb_prune_pairs(PairParams P, int64_t groups_cap, const int32_t *__restrict__ sizes, NbCell H, float rin2,
                   const int2 *__restrict__ slab, const int32_t *__restrict__ counts,
                   const int32_t *__restrict__ order, const float4 *__restrict__ xq,
                   const int32_t *__restrict__ typ, const float2 *__restrict__ lj, const float2 *__restrict__ ljf,
                   int2 *__restrict__ slab_in, int32_t *__restrict__ counts_in, const int *gate,
                   const double *__restrict__ x, double *__restrict__ x_prune, int32_t *unit_counter,
                   int2 *__restrict__ units, double *prunes, float4 *__restrict__ acc, int *__restrict__ status,
                   const int *halt) {
  __shared__ float4 s_x[NB_PRUNE_WARPS][2 * NB_GROUP];
  __shared__ float2 s_f[NB_PRUNE_WARPS][2 * NB_GROUP];
  __shared__ int s_t[NB_PRUNE_WARPS][2 * NB_GROUP];
  __shared__ float2 s_lj[LJM == 0 ? NB_MAX_TYPES * NB_MAX_TYPES : 1];
  __shared__ float s_b[NB_PRUNE_WARPS][3][NB_SPARSE_BITS][33];
  int64_t g = blockIdx.x;
  nb_grid_wait();  // the gate and the frames of the kernels before (a chained launch)
  if (halt && *halt) return;
  if (*gate == 0) return;  // no pruning due: the pair kernel after this one does the pairs
  if (g >= groups_cap || g >= sizes[NB_SIZE_GROUPS]) return;
  if (LJM == 0) {
    int nt2 = P.ntypes * P.ntypes;
    for (int k = threadIdx.x; k < nt2; k += blockDim.x) {
      float2 c = lj[k];
      s_lj[k] = make_float2(6.f * c.x, 12.f * c.y);
    }
  }
  int total = nb_prune_group(g, H, rin2, P.list_cap, slab, counts, order, xq, slab_in, counts_in, x, x_prune,
                             unit_counter, units, P.units_cap, prunes);
  __syncthreads();  // the block's inner list and its count, written to global memory, and s_lj
  int warp = threadIdx.x >> 5;
  int nu = (total + NB_UNIT - 1) / NB_UNIT;
  for (int o = warp; o < nu; o += NB_PRUNE_WARPS)
    nb_pair_unit<false, false, SWITCH, LJM, false>(P, make_int2((int)g, o), 0, make_int2(0, 0), make_int2(0, 0),
                                                   nullptr, slab_in, counts_in, xq, nullptr, nullptr, typ, ljf, s_lj,
                                                   s_x[warp], s_f[warp], s_t[warp], s_b[warp], acc, nullptr,
                                                   nullptr, status);
}

// Frames: xq[p] = ((float)(x_a + (S_p - 1/2) L), q_a) for the atom a at place p;
// an empty place gets zeros (no bit names it).
__global__ void nb_gather(int64_t places, const int32_t *__restrict__ sizes,
                          const int32_t *__restrict__ order, const char4 *__restrict__ shift,
                          const double *__restrict__ x, const float *__restrict__ q,
                          const int32_t *__restrict__ type, double Lx, double Ly, double Lz, double bx,
                          double cx, double cy, float4 *__restrict__ xq, int32_t *__restrict__ typ_p,
                          float4 *__restrict__ xq_lo, const double *__restrict__ cot, float4 *__restrict__ gp) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= places || p >= sizes[NB_SIZE_PLACES]) return;
  int a = order[p];
  if (a < 0) {
    xq[p] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (xq_lo) xq_lo[p] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (gp) gp[p] = make_float4(0.f, 0.f, 0.f, 0.f);
    typ_p[p] = 0;
    return;
  }
  // with cot, the cotangent on the forces (the adjoint's g, f32 per place)
  if (gp) gp[p] = make_float4((float)cot[3 * a], (float)cot[3 * a + 1], (float)cot[3 * a + 2], 0.f);
  // x + S H less half the diagonal (a triclinic cell adds S's tilt terms),
  // and with xq_lo the f32 residual of each coordinate
  char4 s = shift[p];
  // each product and sum rounded once, in this order (no contraction), as
  // the MD step's update makes the frames of the next step (md_frame)
  double fx = __dadd_rn(__dadd_rn(__dadd_rn(x[3 * a], __dmul_rn(nb_frame_shift(s.x), Lx)), __dmul_rn((double)s.y, bx)),
                        __dmul_rn((double)s.z, cx));
  double fy = __dadd_rn(__dadd_rn(x[3 * a + 1], __dmul_rn(nb_frame_shift(s.y), Ly)), __dmul_rn((double)s.z, cy));
  double fz = __dadd_rn(x[3 * a + 2], __dmul_rn(nb_frame_shift(s.z), Lz));
  float4 hi = make_float4((float)fx, (float)fy, (float)fz, q[a]);
  xq[p] = hi;
  if (xq_lo)
    xq_lo[p] = make_float4((float)(fx - (double)hi.x), (float)(fy - (double)hi.y), (float)(fz - (double)hi.z), 0.f);
  typ_p[p] = type[a];
}

// One excluded pair (i < j): the correction -f q_i q_j erf(beta r)/r in the
// minimum image, in f64 from the f32 frames; adds the forces and returns the
// energy and virial in v[0..6].
template <bool FIXED>
__device__ __forceinline__ void nb_excluded_pair(int i, int j, const int32_t *__restrict__ place_of,
                                                 const float4 *__restrict__ xq, double Lx, double Ly, double Lz,
                                                 double bx, double cx, double cy,
                                                 double beta, double coulomb, float4 *__restrict__ acc,
                                                 unsigned long long *__restrict__ accf, int *__restrict__ status,
                                                 double *v) {
  int pi = place_of[i], pj = place_of[j];
  if (pi < 0 || pj < 0) return;
  float4 a = xq[pi], b = xq[pj];
  double d0 = (double)a.x - b.x, d1 = (double)a.y - b.y, d2 = (double)a.z - b.z;
  // the minimum image in one pass along c, b, a (per axis without tilts)
  double nc = rint(d2 / Lz);
  d0 -= nc * cx;
  d1 -= nc * cy;
  d2 -= Lz * nc;
  double nbv = rint(d1 / Ly);
  d0 -= nbv * bx;
  d1 -= Ly * nbv;
  d0 -= Lx * rint(d0 / Lx);
  double r2 = d0 * d0 + d1 * d1 + d2 * d2;
  double qq = coulomb * (double)a.w * (double)b.w;
  if (qq == 0.0 || r2 <= 0.0) return;
  double r = sqrt(r2);
  double ef = erf(beta * r);
  double g = 2.0 * beta / sqrt(M_PI) * exp(-beta * beta * r2);
  double fs = qq * (g / r2 - ef / (r2 * r));
  float fx = (float)(fs * d0), fy = (float)(fs * d1), fz = (float)(fs * d2);
  if (FIXED) {
    nb_red_fixed(accf + 3 * (int64_t)pi, fx, fy, fz, status);
    nb_red_fixed(accf + 3 * (int64_t)pj, -fx, -fy, -fz, status);
  } else {
    nb_red_add_v4(acc + pi, fx, fy, fz);
    nb_red_add_v4(acc + pj, -fx, -fy, -fz);
  }
  v[0] = -qq * ef / r;
  v[1] = d0 * fs * d0;
  v[2] = d1 * fs * d1;
  v[3] = d2 * fs * d2;
  v[4] = d0 * fs * d1;
  v[5] = d0 * fs * d2;
  v[6] = d1 * fs * d2;
}

// The block's sums of v[0..6] to partials[blockIdx.x * 8 + c].
__device__ __forceinline__ void nb_block_partials8(double *v, double *__restrict__ partials) {
  __shared__ double s_part[8][8];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[c] += __shfl_xor_sync(0xffffffffu, v[c], o);
  }
  if (lane == 0)
    for (int c = 0; c < 8; ++c) s_part[warp][c] = v[c];
  __syncthreads();
  if (threadIdx.x < 8) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += s_part[w][threadIdx.x];
    partials[(int64_t)blockIdx.x * 8 + threadIdx.x] = s;
  }
}

// The excluded-pair correction, a thread per pair i < j.
template <bool FIXED>
__global__ void nb_excluded(int64_t npairs, const int32_t *__restrict__ pairs,
                            const int32_t *__restrict__ place_of, const float4 *__restrict__ xq,
                            double Lx, double Ly, double Lz, double bx, double cx, double cy, double beta,
                            double coulomb, bool energy,
                            float4 *__restrict__ acc, unsigned long long *__restrict__ accf,
                            double *__restrict__ partials, int *__restrict__ status) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (k < npairs)
    nb_excluded_pair<FIXED>(pairs[2 * k], pairs[2 * k + 1], place_of, xq, Lx, Ly, Lz, bx, cx, cy, beta, coulomb,
                            acc, accf, status, v);
  if (!energy) return;
  nb_block_partials8(v, partials);
}

// The same over the frames of a batch: block b takes pairs
// [blk_first[b], frame_end[f]) of one frame f = blk_frame[b] (at most 256),
// so that its partial sums belong to one frame.
__global__ void nb_batch_excluded(const int32_t *__restrict__ blk_frame, const int32_t *__restrict__ blk_first,
                                  const int32_t *__restrict__ frame_end, const int32_t *__restrict__ pairs,
                                  const int32_t *__restrict__ place_of, const float4 *__restrict__ xq,
                                  const NbFrameDev *__restrict__ frames, double beta, double coulomb, bool energy,
                                  float4 *__restrict__ acc, double *__restrict__ partials) {
  int f = blk_frame[blockIdx.x];
  int64_t k = (int64_t)blk_first[blockIdx.x] + threadIdx.x;
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (k < frame_end[f]) {
    const NbFrameDev &F = frames[f];
    nb_excluded_pair<false>(pairs[2 * k], pairs[2 * k + 1], place_of, xq, F.L0, F.L1, F.L2, 0.0, 0.0, 0.0, beta,
                            coulomb, acc, nullptr, nullptr, v);
  }
  if (!energy) return;
  nb_block_partials8(v, partials);
}

// Frames of a batch: each place's atom in its frame's cell.
__global__ void nb_batch_gather(int64_t places, const int32_t *__restrict__ sizes,
                                const int32_t *__restrict__ order, const char4 *__restrict__ shift,
                                const double *__restrict__ x, const float *__restrict__ q,
                                const int32_t *__restrict__ type, const int32_t *__restrict__ atom_frame,
                                const NbFrameDev *__restrict__ frames, float4 *__restrict__ xq,
                                int32_t *__restrict__ typ_p) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= places || p >= sizes[NB_SIZE_PLACES]) return;
  int a = order[p];
  if (a < 0) {
    xq[p] = make_float4(0.f, 0.f, 0.f, 0.f);
    typ_p[p] = 0;
    return;
  }
  const NbFrameDev &F = frames[atom_frame[a]];
  char4 s = shift[p];
  xq[p] = make_float4((float)(x[3 * a] + nb_frame_shift(s.x) * F.L0),
                      (float)(x[3 * a + 1] + nb_frame_shift(s.y) * F.L1),
                      (float)(x[3 * a + 2] + nb_frame_shift(s.z) * F.L2), q[a]);
  typ_p[p] = type[a];
}

// The energies and virials of each frame (a block a frame), summed in a
// fixed order: the units of its pairs, the blocks of its excluded pairs and
// of its convolution.
__global__ void nb_batch_sums(int nframes, const int32_t *__restrict__ frame_units,
                              const double *__restrict__ unit_partials, int pairs,
                              const int32_t *__restrict__ excl_blk0, const double *__restrict__ excl_part,
                              int excluded, const int32_t *__restrict__ conv_blk0,
                              const double *__restrict__ conv_part, int pme, double *__restrict__ frame_energy) {
  __shared__ double s[128][8];
  int f = blockIdx.x;
  if (f >= nframes) return;
  double *out = frame_energy + (int64_t)f * NB_E_SLOTS;
  for (int part = 0; part < 3; ++part) {
    int width = part == 2 ? 7 : 8;
    const double *src = part == 0 ? unit_partials : part == 1 ? excl_part : conv_part;
    bool on = part == 0 ? pairs : part == 1 ? excluded : pme;
    int lo = 0, hi = 0;
    if (on) {
      if (part == 0) {
        lo = frame_units[2 * f];
        hi = frame_units[2 * f + 1];
      } else if (part == 1) {
        lo = excl_blk0[f];
        hi = excl_blk0[f + 1];
      } else {
        lo = conv_blk0[f];
        hi = conv_blk0[f + 1];
      }
    }
    double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int r = lo + (int)threadIdx.x; r < hi; r += blockDim.x)
      for (int k = 0; k < width; ++k) v[k] += src[(int64_t)r * width + k];
    for (int k = 0; k < 8; ++k) s[threadIdx.x][k] = v[k];
    __syncthreads();
    for (int stride = blockDim.x / 2; stride > 0; stride >>= 1) {
      if ((int)threadIdx.x < stride)
        for (int k = 0; k < 8; ++k) s[threadIdx.x][k] += s[threadIdx.x + stride][k];
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      if (part == 0) {
        out[NB_E_LJ] = s[0][0];
        out[NB_E_COUL] = s[0][1];
        for (int k = 0; k < 6; ++k) out[NB_W_PAIR + k] = s[0][2 + k];
      } else if (part == 1) {
        out[NB_E_EXCL] = s[0][0];
        for (int k = 0; k < 6; ++k) out[NB_W_PAIR + k] += s[0][1 + k];
      } else {
        out[NB_E_REC] = s[0][0];
        for (int k = 0; k < 6; ++k) out[NB_W_REC + k] = s[0][1 + k];
      }
    }
    __syncthreads();
  }
}

// forces[a] (f64, atom order) = (or +=) the sum of the place accumulators
// of the pairs, the excluded pairs and PME; the accumulators are cleared
// for the next evaluation.
template <bool FIXED>
__global__ void nb_finish(int64_t places, const int32_t *__restrict__ sizes,
                          const int32_t *__restrict__ order, float4 *__restrict__ acc,
                          unsigned long long *__restrict__ accf, const float4 *__restrict__ pme_force,
                          double *__restrict__ forces, int accumulate) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= places || p >= sizes[NB_SIZE_PLACES]) return;
  int a = order[p];
  double f0, f1, f2;
  if (FIXED) {
    long long x = (long long)accf[3 * p], y = (long long)accf[3 * p + 1], z = (long long)accf[3 * p + 2];
    accf[3 * p] = 0ull;
    accf[3 * p + 1] = 0ull;
    accf[3 * p + 2] = 0ull;
    f0 = (double)x * NB_FORCE_SCALE_INV;
    f1 = (double)y * NB_FORCE_SCALE_INV;
    f2 = (double)z * NB_FORCE_SCALE_INV;
  } else {
    float4 v = acc[p];
    acc[p] = make_float4(0.f, 0.f, 0.f, 0.f);
    f0 = v.x;
    f1 = v.y;
    f2 = v.z;
  }
  if (pme_force) {
    float4 w = pme_force[p];
    f0 += w.x;
    f1 += w.y;
    f2 += w.z;
  }
  if (a < 0) return;
  if (accumulate) {
    forces[3 * a] += f0;
    forces[3 * a + 1] += f1;
    forces[3 * a + 2] += f2;
  } else {
    forces[3 * a] = f0;
    forces[3 * a + 1] = f1;
    forces[3 * a + 2] = f2;
  }
}

// Fixed-order sums of per-unit (and per-block) partials: one block, each
// thread a strided run of rows, then a tree.
__global__ void nb_sum_partials(const double *__restrict__ unit_partials,
                                const int32_t *__restrict__ sizes, int64_t units_cap,
                                const double *__restrict__ excl_partials, int excl_blocks,
                                int do_pairs, double *__restrict__ energy) {
  __shared__ double s[256][8];
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  double w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (do_pairs) {
    int64_t nunits = min((int64_t)sizes[NB_SIZE_UNITS], units_cap);
    for (int64_t u = threadIdx.x; u < nunits; u += blockDim.x)
      for (int k = 0; k < 8; ++k) v[k] += unit_partials[u * 8 + k];
  }
  for (int64_t b = threadIdx.x; b < excl_blocks; b += blockDim.x)
    for (int k = 0; k < 8; ++k) w[k] += excl_partials[b * 8 + k];
  // pairs: lj, coul, W(6); excluded: e, W(6): combine W of both in slots
  for (int k = 0; k < 8; ++k) s[threadIdx.x][k] = v[k];
  __syncthreads();
  for (int stride = blockDim.x / 2; stride > 0; stride >>= 1) {
    if ((int)threadIdx.x < stride)
      for (int k = 0; k < 8; ++k) s[threadIdx.x][k] += s[threadIdx.x + stride][k];
    __syncthreads();
  }
  double pv[8];
  for (int k = 0; k < 8; ++k) pv[k] = s[0][k];
  __syncthreads();
  for (int k = 0; k < 8; ++k) s[threadIdx.x][k] = w[k];
  __syncthreads();
  for (int stride = blockDim.x / 2; stride > 0; stride >>= 1) {
    if ((int)threadIdx.x < stride)
      for (int k = 0; k < 8; ++k) s[threadIdx.x][k] += s[threadIdx.x + stride][k];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (do_pairs) {
      energy[NB_E_LJ] = pv[0];
      energy[NB_E_COUL] = pv[1];
    }
    if (excl_blocks > 0) energy[NB_E_EXCL] = s[0][0];
    for (int k = 0; k < 6; ++k)
      energy[NB_W_PAIR + k] = (do_pairs ? pv[2 + k] : 0.0) + (excl_blocks > 0 ? s[0][1 + k] : 0.0);
  }
}

// ---------------------------------------------------------------------------
// The parameter gradient (the differentiation form).
//
// MODE 0, the force-matching product.  With g_i the cotangent on the forces
// (for a loss (1/K) sum |F - F^ref|^2, g = (2/K)(F - F^ref)) and u(r; theta)
// the energy of a pair, F_i = -sum_j u'(r_ij) d_ij / r_ij, so that
//   G_theta = sum_i g_i . dF_i/dtheta = -sum_pairs h_ij du'/dtheta,
//   h_ij = (g_i - g_j) . d_ij / r_ij,
// which gives, with D = d/dr [erfc(beta r)/r] and u_LJ = 4 eps ((sigma/r)^12 - (sigma/r)^6),
//   G_q[i] -= h f q_j D,  G_q[j] -= h f q_i D,
//   G_sigma[ab] -= h 4 eps (36 s6 - 144 s12)/(sigma r),  G_eps[ab] -= h 4 (6 s6 - 12 s12)/r.
// MODE 1, the gradient of the energy:
//   G_q[i] += f q_j (erfc(beta r)/r - shift),  G_sigma[ab] += 4 eps (12 s12 - 6 s6)/sigma,
//   G_eps[ab] += 4 (s12 - s6).
// The kernel walks the same lists and slots as nb_pairs and recomputes the
// geometry (nothing of the forward pass is stored).  The member's G_q
// travels with it like its force accumulator; the partner's stays in its
// lane and is added once per entry (f64 atomics); the type-pair sums go to
// shared memory and are added to per-block partials (the frames of a call
// accumulate there), summed later in a fixed order.  The shared table holds
// (sigma, eps/sigma) per type pair, so the sigma term needs no division.
// MDIR's counterpart is the IR-derived product of md-differentiate (D381,
// docs/python-frames.md:203-260), which walks the neighbor matrix.
// Warps a block of the adjoint kernel: one, so that a warp that finishes
// early (each takes a fixed share of units) frees its place on the SM for
// the kernels of the other frames running beside it at once, rather than
// wait at the block's barrier (1, 2, 4 and 8 measured 2.78-2.81, 2.82-2.86,
// 2.84-2.87 and 2.93 ms for the product of 64 frames on four lanes).
#ifndef NB_ADJ_WARPS
#define NB_ADJ_WARPS 1
#endif

template <int MODE>
__global__ void __launch_bounds__(NB_ADJ_WARPS * 32, 32 / NB_ADJ_WARPS) nb_pairs_adjoint(
    PairParams P, const int32_t *__restrict__ sizes, const int2 *__restrict__ units, const int2 *__restrict__ slab,
    const int32_t *__restrict__ counts, const float4 *__restrict__ xq, const int32_t *__restrict__ typ,
    const float2 *__restrict__ sigeps, const float4 *__restrict__ gp, double *__restrict__ gq,
    double *__restrict__ type_partials, const int32_t *__restrict__ counts_lj) {
  __shared__ float4 s_x[NB_ADJ_WARPS][2 * NB_GROUP];
  __shared__ float4 s_g[NB_ADJ_WARPS][2 * NB_GROUP];  // the cotangent, and in w the member's type row (ntypes t)
  // (sigma, eps/sigma) per type pair, then the 2 ntypes^2 sums (dynamic: ntypes^2 x 16 bytes)
  extern __shared__ float2 s_dyn[];
  const unsigned FULL = 0xffffffffu;
  int nt2 = P.ntypes * P.ntypes;
  float2 *s_se = s_dyn;
  float *s_acc = reinterpret_cast<float *>(s_dyn + nt2);
  for (int k = threadIdx.x; k < nt2; k += blockDim.x) {
    float2 se = sigeps[k];
    s_se[k] = make_float2(se.x, se.x > 0.f ? se.y / se.x : 0.f);
    s_acc[k] = 0.f;
    s_acc[nt2 + k] = 0.f;
  }
  __syncthreads();
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int u = lane & 15;
  const int src = (lane & 16) | ((lane + 1) & 15);
  const float4 *px = &s_x[warp][u];
  const float4 *pg = &s_g[warp][u];
  int nunits = min((int64_t)sizes[NB_SIZE_UNITS], P.units_cap);
  int wstride = gridDim.x * NB_ADJ_WARPS;
  for (int unit = blockIdx.x * NB_ADJ_WARPS + warp; unit < nunits; unit += wstride) {
    int2 uo = units[unit];
    int g = uo.x;
    int64_t pi = (int64_t)g * NB_GROUP + u;
    __syncwarp();
    {
      float4 xi = xq[pi];
      xi.w *= P.coulomb;
      s_x[warp][lane] = xi;
      float4 gi = MODE == 0 ? gp[pi] : make_float4(0.f, 0.f, 0.f, 0.f);
      gi.w = __int_as_float(typ[pi] * P.ntypes);
      s_g[warp][lane] = gi;
    }
    __syncwarp();
    int cnt = (int)min((int64_t)counts[g], P.list_cap);
    int e0 = uo.y * NB_UNIT;
    int ne = min(NB_UNIT, cnt - e0);
    // with the lists partitioned (counts_lj), the rounds that start past a
    // group's LJ partners have none (the same for the whole warp)
    int nlj = counts_lj ? counts_lj[g] : cnt;
    float ai = 0.f;  // G_q of member (lane + k) mod 16
    for (int r = 0; r < 2; ++r) {
      if (r * 32 >= ne) break;
      const bool lj_round = e0 + r * 32 < nlj;
      bool valid = r * 32 + lane < ne;
      int2 en = valid ? slab[(int64_t)g * P.list_cap + e0 + r * 32 + lane] : make_int2(0, 0);
      int q = en.x;
      unsigned mask = valid ? ((unsigned)en.y & 0xffffu) : 0u;
      int code = ((unsigned)en.y >> 16) & NB_IMAGE_BITS;
      int sx, sy, sz;
      nb_decode_image(code, sx, sy, sz);
      float4 xj = xq[q];
      {
        NbCell H;
        H.ax = P.Lx;
        H.by = P.Ly;
        H.cz = P.Lz;
        H.bx = P.bx;
        H.cx = P.cx;
        H.cy = P.cy;
        float3 t = nb_lattice_shift(sx, sy, sz, H);
        xj.x += t.x;
        xj.y += t.y;
        xj.z += t.z;
      }
      float4 gj = MODE == 0 ? gp[q] : make_float4(0.f, 0.f, 0.f, 0.f);
      int tj = typ[q];
      float fqj = xj.w * P.coulomb;
      unsigned mrot = ((mask >> u) | (mask << (16 - u))) & 0xffffu;
      float aj = 0.f;
#pragma unroll 4
      for (int k = 0; k < NB_GROUP; ++k) {
        float4 xm = px[k];
        float dx = xm.x - xj.x, dy = xm.y - xj.y, dz = xm.z - xj.z;
        float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        bool inside = ((mrot >> k) & 1u) && (r2 < P.rc2);
        float r2s = inside ? r2 : 1.0f;
        float rinv = nb_rsqrt(r2s);
        float rinv2 = rinv * rinv;
        float rr = r2s * rinv;
        float ex = nb_ex2(r2s * P.nb2_log2e);
        float erfcv = nb_erfc_from_exp(P.beta_p * rr, ex);
        // w: the factor of the pair's term; cq: its Coulomb part per unit f q_i q_j
        float w, cq;
        float4 gm = pg[k];
        if (MODE == 0) {
          float h = ((gm.x - gj.x) * dx + (gm.y - gj.y) * dy + (gm.z - gj.z) * dz) * rinv;
          w = inside ? h : 0.f;
          // -h D, D = -(erfc(beta r)/r^2 + 2 beta/sqrt(pi) exp(-beta^2 r^2)/r)
          cq = w * fmaf(erfcv, rinv2, P.two_beta_sqrtpi * ex * rinv);
        } else {
          w = inside ? 1.f : 0.f;
          cq = w * (erfcv * rinv - P.coulomb_shift);
        }
        ai = fmaf(cq, fqj, ai);
        aj = fmaf(cq, xm.w, aj);
        if (lj_round && w != 0.f) {
          int tp = __float_as_int(gm.w) + tj;
          float2 se = s_se[tp];  // (sigma, eps / sigma)
          if (se.y != 0.f) {
          float s1 = se.x * rinv;
          float s2 = s1 * s1;
          float s6 = s2 * s2 * s2;
          float s12 = s6 * s6;
          float ds, de;
          if (MODE == 0) {
            float a = -4.f * w * rinv;
            de = a * (6.f * s6 - 12.f * s12);
            ds = a * se.y * (36.f * s6 - 144.f * s12);
          } else {
            de = 4.f * (s12 - s6);
            ds = 4.f * se.y * (12.f * s12 - 6.f * s6);
          }
          atomicAdd(&s_acc[tp], ds);
          atomicAdd(&s_acc[nt2 + tp], de);
          }
        }
        ai = __shfl_sync(FULL, ai, src);
      }
      if (valid && aj != 0.f) atomicAdd(gq + q, (double)aj);
    }
    ai += __shfl_xor_sync(FULL, ai, 16);
    if (lane < 16 && ai != 0.f) atomicAdd(gq + pi, (double)ai);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < 2 * nt2; k += blockDim.x)
    type_partials[(int64_t)blockIdx.x * 2 * nt2 + k] += (double)s_acc[k];
}

// The per-place charge gradient (f64) added to atom order; the place
// values are zeroed for the next call.
__global__ void nb_scatter_place_values(int64_t places, const int32_t *__restrict__ sizes,
                                        const int32_t *__restrict__ order, double *__restrict__ vp,
                                        double *__restrict__ out) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= places) return;
  double v = vp[p];
  if (v != 0.0) {
    int a = p < sizes[NB_SIZE_PLACES] ? order[p] : -1;
    if (a >= 0) out[a] += v;
    vp[p] = 0.0;
  }
}

// The stable partition of each group's list by the partner's LJ terms: the
// entries whose partner's type has any, then the others, each in their
// order; counts_lj[g] gets the number of the first.  One warp a group, its
// entries staged in shared memory (list_cap of them).
__global__ void __launch_bounds__(32) nb_lj_partition(const int32_t *__restrict__ sizes, int64_t list_cap,
                                                      const int32_t *__restrict__ counts, int2 *__restrict__ slab,
                                                      const int32_t *__restrict__ order,
                                                      const int32_t *__restrict__ type,
                                                      const int32_t *__restrict__ lj_on,
                                                      int32_t *__restrict__ counts_lj) {
  extern __shared__ int2 s_e[];
  int64_t g = blockIdx.x;
  if (g >= sizes[NB_SIZE_GROUPS]) return;
  int lane = threadIdx.x;
  int cnt = (int)min((int64_t)counts[g], list_cap);
  int2 *row = slab + g * list_cap;
  for (int e = lane; e < cnt; e += 32) s_e[e] = row[e];
  __syncwarp();
  auto lj = [&](int e) {
    int a = order[s_e[e].x];
    return a >= 0 && lj_on[type[a]] != 0;
  };
  int nlj = 0;
  for (int e0 = 0; e0 < cnt; e0 += 32) nlj += __popc(__ballot_sync(0xffffffffu, e0 + lane < cnt && lj(e0 + lane)));
  int pl = 0, pn = nlj;
  unsigned below = (1u << lane) - 1u;
  for (int e0 = 0; e0 < cnt; e0 += 32) {
    int e = e0 + lane;
    bool in = e < cnt;
    bool f = in && lj(e);
    unsigned bl = __ballot_sync(0xffffffffu, f);
    unsigned bn = __ballot_sync(0xffffffffu, in && !f);
    if (in) row[f ? pl + __popc(bl & below) : pn + __popc(bn & below)] = s_e[e];
    pl += __popc(bl);
    pn += __popc(bn);
  }
  if (lane == 0) counts_lj[g] = nlj;
}

// The excluded pairs, u = -f q_i q_j erf(beta r)/r, in f64 and atom order.
// MODE 0: G_q[i] += h f q_j X, X = d/dr [erf(beta r)/r]; MODE 1: G_q[i] -= f q_j erf(beta r)/r.
template <int MODE>
__global__ void nb_excluded_adjoint(int64_t npairs, const int32_t *__restrict__ pairs, const double *__restrict__ x,
                                    const float *__restrict__ q, const double *__restrict__ g, double Lx, double Ly,
                                    double Lz, double beta, double coulomb, double *__restrict__ gq) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= npairs) return;
  int i = pairs[2 * k], j = pairs[2 * k + 1];
  double d0 = x[3 * i] - x[3 * j], d1 = x[3 * i + 1] - x[3 * j + 1], d2 = x[3 * i + 2] - x[3 * j + 2];
  d0 -= Lx * rint(d0 / Lx);
  d1 -= Ly * rint(d1 / Ly);
  d2 -= Lz * rint(d2 / Lz);
  double r2 = d0 * d0 + d1 * d1 + d2 * d2;
  if (r2 <= 0.0) return;
  double r = sqrt(r2);
  double c;
  if (MODE == 0) {
    double h = ((g[3 * i] - g[3 * j]) * d0 + (g[3 * i + 1] - g[3 * j + 1]) * d1 + (g[3 * i + 2] - g[3 * j + 2]) * d2) / r;
    double X = 2.0 * beta / sqrt(M_PI) * exp(-beta * beta * r2) / r - erf(beta * r) / r2;
    c = h * coulomb * X;
  } else {
    c = -coulomb * erf(beta * r) / r;
  }
  atomicAdd(gq + i, c * (double)q[j]);
  atomicAdd(gq + j, c * (double)q[i]);
}

// The charge terms of the energy without a pair: the Ewald self term
// -f beta/sqrt(pi) sum q^2 and the neutralizing background -f pi Q^2/(2 V beta^2).
__global__ void nb_charge_terms(int64_t n, const float *__restrict__ q, double self2, double background,
                                double *__restrict__ gq) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  gq[i] += self2 * (double)q[i] + background;
}

// Fixed-order sum of the per-block type-pair partials, added into out: a
// block of NB_SUM_THREADS per value, thread t summing blocks t, t + 256, ...
// in turn, then the threads by a fixed tree (the same order every call).
// The partials are block-major (each adjoint block writes its row whole).
#define NB_SUM_THREADS 256
__global__ void __launch_bounds__(NB_SUM_THREADS) nb_sum_type_partials(const double *__restrict__ partials,
                                                                      int nblocks, int width,
                                                                      double *__restrict__ out) {
  __shared__ double s_sum[NB_SUM_THREADS / 32];
  const int k = blockIdx.x, t = threadIdx.x;
  double s = 0.0;
  for (int b = t; b < nblocks; b += NB_SUM_THREADS) s += partials[(int64_t)b * width + k];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((t & 31) == 0) s_sum[t >> 5] = s;
  __syncthreads();
  if (t == 0) {
    double total = 0.0;
    for (int w = 0; w < NB_SUM_THREADS / 32; ++w) total += s_sum[w];
    out[k] += total;
  }
}

inline int blocks_for(int64_t n, int t) { return (int)std::max<int64_t>(1, (n + t - 1) / t); }

int g_sm_count = 0;

void ensure_sm_count() {
  if (!g_sm_count) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
    if (g_sm_count <= 0) g_sm_count = 148;
  }
}

PairParams pair_params(const NbCtx &c, const double box[3]) {
  PairParams P;
  P.update_after = 0;
  P.Lx = (float)box[0];
  P.Ly = (float)box[1];
  P.Lz = (float)box[2];
  P.bx = (float)c.tilt[0];
  P.cx = (float)c.tilt[1];
  P.cy = (float)c.tilt[2];
  P.Ld[0] = box[0];
  P.Ld[1] = box[1];
  P.Ld[2] = box[2];
  P.Ld[3] = c.tilt[0];
  P.Ld[4] = c.tilt[1];
  P.Ld[5] = c.tilt[2];
  P.rc2 = (float)(c.cutoff * c.cutoff);
  P.beta = (float)c.beta;
  P.beta_p = (float)(0.3275911 * c.beta);
  P.nb2_log2e = (float)(-c.beta * c.beta / log(2.0));
  P.two_beta_sqrtpi = (float)(2.0 * c.beta / sqrt(M_PI));
  P.coulomb = (float)c.coulomb;
  P.coulomb_shift = c.coulomb_shift ? (float)(erfc(c.beta * c.cutoff) / c.cutoff) : 0.f;
  double rs2 = c.switch_distance * c.switch_distance;
  P.rs2 = (float)rs2;
  P.winv = c.lj_switch == 1 ? (float)(1.0 / (c.cutoff * c.cutoff - rs2)) : 0.f;
  P.rs = (float)c.switch_distance;
  P.winv_r = c.lj_switch == 2 ? (float)(1.0 / (c.cutoff - c.switch_distance)) : 0.f;
  P.ntypes = c.ntypes;
  P.list_cap = c.list_cap;
  P.units_cap = c.units_cap;
  return P;
}

}  // namespace

void nb_gather_frames(NbCtx &c, const double *x, const double box[3], cudaStream_t s, const double *cot) {
  nb_gather<<<blocks_for(c.places_cap, 256), 256, 0, s>>>(c.places_cap, c.sizes, c.order, c.shift, x,
                                                          c.q, c.type, box[0], box[1], box[2], c.tilt[0],
                                                          c.tilt[1], c.tilt[2], c.xq, c.typ_p,
                                                          c.deterministic ? c.xq_lo : nullptr, cot,
                                                          cot ? c.adj_g : nullptr);
}

bool nb_fused_prune(const NbCtx &c) {
  if (c.deterministic || !(c.inner_reach > 0.0) || sizeof(int2) * (size_t)c.list_cap > NB_FUSED_STAGE_MAX)
    return false;
  if (c.fused_prune == 1) return true;
  if (c.fused_prune == 2) return false;
  return c.h_sizes && c.h_sizes[NB_SIZE_GROUPS] >= NB_FUSED_PRUNE_GROUPS;
}

void nb_prune_pairs_run(NbCtx &c, const double box[3], const int *gate, const double *x, double *x_prune,
                        double *prunes, int32_t *unit_counter, cudaStream_t s, const int *halt) {
  PairParams P = pair_params(c, box);
  double Rw = c.inner_reach + 3e-6 * (box[0] + box[1] + box[2] + fabs(c.tilt[0]) + fabs(c.tilt[1]) + fabs(c.tilt[2]));
  size_t stage = sizeof(int2) * (size_t)c.list_cap;
  NbCell H = nb_cell(c, box);
#define NB_FUSED_LAUNCH(S, M)                                                                                    \
  do {                                                                                                          \
    static size_t configured[64] = {};                                                                          \
    int dev = 0;                                                                                                \
    cudaGetDevice(&dev);                                                                                        \
    if (dev >= 0 && dev < 64 && configured[dev] < stage) {                                                       \
      cudaFuncSetAttribute(nb_prune_pairs<S, M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage);      \
      configured[dev] = stage;                                                                                  \
    }                                                                                                           \
    nb_launch_chained(nb_prune_pairs<S, M>, dim3((int)c.groups_cap), dim3(NB_PRUNE_WARPS * 32), stage, s, P,     \
                      c.groups_cap, c.sizes, H, (float)(Rw * Rw), c.slab, c.counts, c.order, c.xq, c.typ_p,    \
                      c.lj, c.ljf, c.slab_in, c.counts_in, gate, x, x_prune, unit_counter, c.units_in, prunes,   \
                      c.acc, c.status, halt);                                                                   \
  } while (0)
#define NB_FUSED_M(S)           \
  do {                          \
    if (c.lj_geom)              \
      NB_FUSED_LAUNCH(S, 1);    \
    else                        \
      NB_FUSED_LAUNCH(S, 0);    \
  } while (0)
  if (c.lj_switch == 2)
    NB_FUSED_M(2);
  else if (c.lj_switch == 1)
    NB_FUSED_M(1);
  else
    NB_FUSED_M(0);
#undef NB_FUSED_M
#undef NB_FUSED_LAUNCH
}

void nb_pairs_run(NbCtx &c, const double box[3], bool energy, cudaStream_t s, const int *halt, const int *skip,
                  bool update_after) {
  ensure_sm_count();
  PairParams P = pair_params(c, box);
  P.update_after = update_after ? 1 : 0;
  // persistent grid: enough warps for the units, `pair_blocks_per_sm`
  // blocks of 8 warps per SM (4 fit at 64 registers; fewer leave room for
  // the PME kernels that run beside it on another stream)
  int64_t want = (c.units_cap + NB_PAIR_WARPS - 1) / NB_PAIR_WARPS;
  int sms = c.pair_sms > 0 ? std::min(c.pair_sms, g_sm_count) : g_sm_count;
  int grid = (int)std::min<int64_t>(want, (int64_t)sms * std::max(1, c.pair_blocks_per_sm) * (8 / NB_PAIR_WARPS));
  if (grid < 1) grid = 1;
  // the inner list of the dual list once it has been pruned, else the outer
  bool inner = c.inner_reach > 0.0 && c.inner_valid;
  const int32_t *lsizes = inner ? c.sizes_in : c.sizes;
  const int2 *lunits = inner ? c.units_in : c.units;
  const int2 *lslab = inner ? c.slab_in : c.slab;
  const int32_t *lcounts = inner ? c.counts_in : c.counts;
#define NB_LAUNCH3(E, F, S, M, D)                                                                          \
  nb_launch_chained(nb_pairs<E, F, S, M, false, D>, dim3(grid), dim3(NB_PAIR_WARPS * 32), 0, s, P,             \
                    (const float4 *)nullptr,                                                                 \
                    lsizes, lunits, lslab, lcounts, c.xq, c.xq_lo, c.typ_p, c.lj, c.ljf, c.acc, c.acc_fixed,  \
                    c.unit_partials, c.status, halt, skip)
#define NB_LAUNCH2(E, F, S, M)                     \
  do {                                             \
    if (c.staging_depth == 2)                      \
      NB_LAUNCH3(E, F, S, M, 2);                   \
    else                                           \
      NB_LAUNCH3(E, F, S, M, 1);                   \
  } while (0)
#define NB_LAUNCH(E, F, S)      \
  do {                          \
    if (c.lj_geom)              \
      NB_LAUNCH2(E, F, S, 1);   \
    else                        \
      NB_LAUNCH2(E, F, S, 0);   \
  } while (0)
#define NB_LAUNCH_S(E, F)        \
  do {                           \
    if (c.lj_switch == 2)        \
      NB_LAUNCH(E, F, 2);        \
    else if (c.lj_switch == 1)   \
      NB_LAUNCH(E, F, 1);        \
    else                         \
      NB_LAUNCH(E, F, 0);        \
  } while (0)
  bool F = c.deterministic;
  if (energy) {
    if (F) NB_LAUNCH_S(true, true); else NB_LAUNCH_S(true, false);
  } else {
    if (F) NB_LAUNCH_S(false, true); else NB_LAUNCH_S(false, false);
  }
#undef NB_LAUNCH_S
#undef NB_LAUNCH
#undef NB_LAUNCH2
#undef NB_LAUNCH3
}

void nb_excluded_list_run(NbCtx &c, const double box[3], const int32_t *pairs, int64_t npairs,
                          cudaStream_t s) {
  if (npairs == 0 || c.beta == 0.0) return;
  int blocks = blocks_for(npairs, 256);
  if (c.deterministic)
    nb_excluded<true><<<blocks, 256, 0, s>>>(npairs, pairs, c.place_of, c.xq, box[0], box[1], box[2], c.tilt[0], c.tilt[1], c.tilt[2], c.beta,
                                             c.coulomb, false, c.acc, c.acc_fixed, nullptr, c.status);
  else
    nb_excluded<false><<<blocks, 256, 0, s>>>(npairs, pairs, c.place_of, c.xq, box[0], box[1], box[2], c.tilt[0], c.tilt[1], c.tilt[2], c.beta,
                                              c.coulomb, false, c.acc, c.acc_fixed, nullptr, c.status);
}

void nb_excluded_run(NbCtx &c, const double box[3], bool energy, cudaStream_t s) {
  if (c.n_excl_pairs == 0 || c.beta == 0.0) return;
  int blocks = blocks_for(c.n_excl_pairs, 256);
  if (c.deterministic)
    nb_excluded<true><<<blocks, 256, 0, s>>>(c.n_excl_pairs, c.excl_pairs, c.place_of, c.xq, box[0],
                                             box[1], box[2], c.tilt[0], c.tilt[1], c.tilt[2], c.beta, c.coulomb, energy, c.acc,
                                             c.acc_fixed, c.excl_partials, c.status);
  else
    nb_excluded<false><<<blocks, 256, 0, s>>>(c.n_excl_pairs, c.excl_pairs, c.place_of, c.xq, box[0],
                                              box[1], box[2], c.tilt[0], c.tilt[1], c.tilt[2], c.beta, c.coulomb, energy, c.acc,
                                              c.acc_fixed, c.excl_partials, c.status);
}

void nb_finish_forces(NbCtx &c, double *forces, int accumulate, cudaStream_t s) {
  const float4 *pf = c.pme.on ? (const float4 *)c.pme.pme_force : nullptr;
  if (c.deterministic)
    nb_finish<true><<<blocks_for(c.places_cap, 256), 256, 0, s>>>(c.places_cap, c.sizes, c.order, c.acc,
                                                                 c.acc_fixed, pf, forces, accumulate);
  else
    nb_finish<false><<<blocks_for(c.places_cap, 256), 256, 0, s>>>(c.places_cap, c.sizes, c.order, c.acc,
                                                                  c.acc_fixed, pf, forces, accumulate);
}

void nb_reduce_energy(NbCtx &c, bool pairs, bool excluded, cudaStream_t s) {
  int eb = (excluded && c.n_excl_pairs > 0 && c.beta != 0.0) ? blocks_for(c.n_excl_pairs, 256) : 0;
  bool inner = c.inner_reach > 0.0 && c.inner_valid;
  nb_sum_partials<<<1, 256, 0, s>>>(c.unit_partials, inner ? c.sizes_in : c.sizes, c.units_cap, c.excl_partials,
                                    eb, pairs ? 1 : 0, c.energy);
}

int nb_adjoint_reserve(NbCtx &c) {
  ensure_sm_count();
  // per block of the adjoint kernel, the 2 ntypes^2 type-pair sums
  int width = 2 * c.ntypes * c.ntypes;
  if (!c.adj_types || c.adj_width < width) {
    if (c.adj_types) cudaFree(c.adj_types);
    c.adj_types = nullptr;
    c.adj_width = 0;
    c.adj_blocks = g_sm_count * (32 / NB_ADJ_WARPS);
    if (cudaMalloc(&c.adj_types, sizeof(double) * c.adj_blocks * width) != cudaSuccess) return -1;
    c.adj_width = width;
  }
  if (c.adj_places < c.places_cap) {
    if (c.adj_g) cudaFree(c.adj_g);
    if (c.adj_q) cudaFree(c.adj_q);
    c.adj_g = nullptr;
    c.adj_q = nullptr;
    c.adj_places = 0;
    if (cudaMalloc(&c.adj_g, sizeof(float4) * c.places_cap) != cudaSuccess) return -1;
    if (cudaMalloc(&c.adj_q, sizeof(double) * c.places_cap) != cudaSuccess) return -1;
    if (cudaMemset(c.adj_q, 0, sizeof(double) * c.places_cap) != cudaSuccess) return -1;
    c.adj_places = c.places_cap;
  }
  return 0;
}

int nb_lj_partition_run(NbCtx &c, cudaStream_t s) {
  c.lj_part_build = -1;
  size_t stage = sizeof(int2) * (size_t)c.list_cap;
  if (c.inner_reach > 0.0 || !c.lj_on || c.groups_cap <= 0 || c.list_cap <= 0 || stage > 227 * 1024) return 0;
  if (stage > 48 * 1024) {
    // the shared-memory opt-in for this list capacity (once per device and size)
    static size_t configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return 0;
    if (configured[dev] < stage) {
      if (cudaFuncSetAttribute(nb_lj_partition, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage) !=
          cudaSuccess)
        return -1;
      configured[dev] = stage;
    }
  }
  if (c.counts_lj_cap < c.groups_cap) {
    if (c.counts_lj) cudaFree(c.counts_lj);
    c.counts_lj = nullptr;
    c.counts_lj_cap = 0;
    if (cudaMalloc(&c.counts_lj, sizeof(int32_t) * c.groups_cap) != cudaSuccess) return -1;
    c.counts_lj_cap = c.groups_cap;
  }
  nb_lj_partition<<<(unsigned)c.groups_cap, 32, stage, s>>>(c.sizes, c.list_cap, c.counts, c.slab, c.order, c.type,
                                                            c.lj_on, c.counts_lj);
  if (cudaGetLastError() != cudaSuccess) return -1;
  c.lj_part_build = c.builds;
  c.lj_part_mask = c.lj_mask;
  return 0;
}

int nb_adjoint_run(NbCtx &c, const double *x, int64_t x_stride, int64_t count, const double box[3],
                   const double *cot, int64_t c_stride, int mode, const float *phi, int64_t p_stride, double *dq,
                   double *dtable, cudaStream_t s) {
  PairParams P = pair_params(c, box);
  bool inner = c.inner_reach > 0.0 && c.inner_valid;
  const int32_t *lsizes = inner ? c.sizes_in : c.sizes;
  const int2 *lunits = inner ? c.units_in : c.units;
  const int2 *lslab = inner ? c.slab_in : c.slab;
  const int32_t *lcounts = inner ? c.counts_in : c.counts;
  int64_t want = (c.units_cap + NB_ADJ_WARPS - 1) / NB_ADJ_WARPS;
  int grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, c.adj_blocks));
  int width = 2 * c.ntypes * c.ntypes;
  size_t smem = sizeof(float2) * c.ntypes * c.ntypes * 2;
  const int32_t *lj_counts =
      !inner && c.lj_part_build == c.builds && c.lj_part_mask == c.lj_mask ? c.counts_lj : nullptr;
  // the blocks' type-pair partials and the places' charge gradient (kept
  // zero between calls) sum the frames; both go out once at the end
  if (cudaMemsetAsync(c.adj_types, 0, sizeof(double) * grid * width, s) != cudaSuccess) return -1;
  double net = 0.0;
  if (mode == 1)
    for (double v : c.h_q) net += v;
  for (int64_t k = 0; k < count; ++k) {
    const double *xk = x + k * x_stride;
    const double *ck = mode == 0 ? cot + k * c_stride : nullptr;
    nb_gather_frames(c, xk, box, s, ck);
    if (mode == 0)
      nb_pairs_adjoint<0><<<grid, NB_ADJ_WARPS * 32, smem, s>>>(P, lsizes, lunits, lslab, lcounts, c.xq, c.typ_p,
                                                                c.sigeps, c.adj_g, c.adj_q, c.adj_types, lj_counts);
    else
      nb_pairs_adjoint<1><<<grid, NB_ADJ_WARPS * 32, smem, s>>>(P, lsizes, lunits, lslab, lcounts, c.xq, c.typ_p,
                                                                c.sigeps, c.adj_g, c.adj_q, c.adj_types, lj_counts);
    int rc = nb_pme_adjoint_run(c, box, mode, s, phi ? phi + k * p_stride : nullptr);
    if (rc) return rc;
    if (c.n_excl_pairs > 0 && c.beta != 0.0) {
      int blocks = blocks_for(c.n_excl_pairs, 256);
      if (mode == 0)
        nb_excluded_adjoint<0><<<blocks, 256, 0, s>>>(c.n_excl_pairs, c.excl_pairs, xk, c.q, ck, box[0], box[1],
                                                      box[2], c.beta, c.coulomb, dq);
      else
        nb_excluded_adjoint<1><<<blocks, 256, 0, s>>>(c.n_excl_pairs, c.excl_pairs, xk, c.q, ck, box[0], box[1],
                                                      box[2], c.beta, c.coulomb, dq);
    }
    if (mode == 1 && c.beta > 0.0) {
      double V = box[0] * box[1] * box[2];
      double self2 = -2.0 * c.coulomb * c.beta / sqrt(M_PI);
      double background = -c.coulomb * M_PI * net / (V * c.beta * c.beta);
      nb_charge_terms<<<blocks_for(c.n, 256), 256, 0, s>>>(c.n, c.q, self2, background, dq);
    }
  }
  nb_sum_type_partials<<<width, NB_SUM_THREADS, 0, s>>>(c.adj_types, grid, width, dtable);
  nb_scatter_place_values<<<blocks_for(c.places_cap, 256), 256, 0, s>>>(c.places_cap, c.sizes, c.order, c.adj_q,
                                                                        dq);
  return 0;
}

// ---------------------------------------------------------------------------
// The batch (mdrtNbBatch): one launch of each kernel over all frames.

void nb_batch_gather_frames(mdrtNbBatch &b, const double *x, cudaStream_t s) {
  NbCtx &c = b.nb->c;
  nb_batch_gather<<<blocks_for(c.places_cap, 256), 256, 0, s>>>(c.places_cap, c.sizes, c.order, c.shift, x, c.q,
                                                                c.type, b.atom_frame, b.frames_dev, c.xq, c.typ_p);
}

void nb_batch_pairs_run(mdrtNbBatch &b, bool energy, cudaStream_t s) {
  NbCtx &c = b.nb->c;
  ensure_sm_count();
  double unit_box[3] = {1.0, 1.0, 1.0};  // the cells come from group_L
  PairParams P = pair_params(c, unit_box);
  int64_t want = (c.units_cap + NB_PAIR_WARPS - 1) / NB_PAIR_WARPS;
  int grid = (int)std::max<int64_t>(
      1, std::min<int64_t>(want, (int64_t)g_sm_count * std::max(1, c.pair_blocks_per_sm) * (8 / NB_PAIR_WARPS)));
#define NB_BATCH_LAUNCH(E, M, D)                                                                               \
  nb_pairs<E, false, 0, M, true, D><<<grid, NB_PAIR_WARPS * 32, 0, s>>>(P, b.group_L, c.sizes, c.units, c.slab, c.counts, c.xq,  \
                                                            nullptr, c.typ_p, c.lj, c.ljf, c.acc, c.acc_fixed,     \
                                                            c.unit_partials, c.status, nullptr, nullptr)
  if (energy) {
    if (c.staging_depth == 2) {
      if (c.lj_geom) NB_BATCH_LAUNCH(true, 1, 2); else NB_BATCH_LAUNCH(true, 0, 2);
    } else {
      if (c.lj_geom) NB_BATCH_LAUNCH(true, 1, 1); else NB_BATCH_LAUNCH(true, 0, 1);
    }
  } else if (c.staging_depth == 2) {
    if (c.lj_geom) NB_BATCH_LAUNCH(false, 1, 2); else NB_BATCH_LAUNCH(false, 0, 2);
  } else {
    if (c.lj_geom) NB_BATCH_LAUNCH(false, 1, 1); else NB_BATCH_LAUNCH(false, 0, 1);
  }
#undef NB_BATCH_LAUNCH
}

void nb_batch_excluded_run(mdrtNbBatch &b, bool energy, cudaStream_t s) {
  NbCtx &c = b.nb->c;
  if (b.excl_blocks == 0 || c.beta == 0.0) return;
  nb_batch_excluded<<<b.excl_blocks, 256, 0, s>>>(b.excl_blk_frame, b.excl_blk_first, b.excl_frame_end,
                                                  c.excl_pairs, c.place_of, c.xq, b.frames_dev, c.beta, c.coulomb,
                                                  energy, c.acc, b.excl_part);
}

void nb_batch_energy_sums(mdrtNbBatch &b, bool pairs, bool excluded, bool pme, cudaStream_t s) {
  NbCtx &c = b.nb->c;
  bool ex = excluded && b.excl_blocks > 0 && c.beta != 0.0;
  cudaMemsetAsync(b.frame_energy, 0, sizeof(double) * NB_E_SLOTS * b.frames, s);
  nb_batch_sums<<<b.frames, 128, 0, s>>>(b.frames, b.frame_units, c.unit_partials, pairs ? 1 : 0, b.d_excl_blk0,
                                         b.excl_part, ex ? 1 : 0, b.d_conv_blk0, b.conv_part, pme ? 1 : 0,
                                         b.frame_energy);
}
