// The pruning of a group's outer list into its inner list (the dual list,
// MDIR D114: emitGroupsPrune, lib/Conversion/MDExecToGPU/MDExecToGPU.cpp:9588;
// docs/neighbor-groups.md Section 6.2), shared by the pruning kernel
// (nb_build.cu) and the pair kernel that prunes on a pruning step
// (nb_pairs.cu; MDIR D284).
#pragma once
#include "nb_common.cuh"

namespace {

// The box of a group's live members, reduced over a warp whose lanes
// 0..15 hold the members (dead lanes and lanes 16..31 give nothing).
__device__ __forceinline__ void nb_live_box(float4 xm, bool on, float3 &lo, float3 &hi) {
  const unsigned FULL = 0xffffffffu;
  lo = on ? make_float3(xm.x, xm.y, xm.z) : make_float3(3.0e38f, 3.0e38f, 3.0e38f);
  hi = on ? make_float3(xm.x, xm.y, xm.z) : make_float3(-3.0e38f, -3.0e38f, -3.0e38f);
  for (int o = 16; o > 0; o >>= 1) {
    lo.x = fminf(lo.x, __shfl_xor_sync(FULL, lo.x, o));
    lo.y = fminf(lo.y, __shfl_xor_sync(FULL, lo.y, o));
    lo.z = fminf(lo.z, __shfl_xor_sync(FULL, lo.z, o));
    hi.x = fmaxf(hi.x, __shfl_xor_sync(FULL, hi.x, o));
    hi.y = fmaxf(hi.y, __shfl_xor_sync(FULL, hi.y, o));
    hi.z = fmaxf(hi.z, __shfl_xor_sync(FULL, hi.z, o));
  }
}

// True when the point lies farther than the pruned reach from the whole box,
// so that no member can pass the member test.  Each axis gap is one member's
// own difference (the box corner is a member coordinate), never more than any
// member's; `far2` = R_in'^2 (1 + 1e-4) covers the rounding of the squares and
// their sum, so the test only drops what the member loop would drop.
__device__ __forceinline__ bool nb_beyond_box(float3 lo, float3 hi, float jx, float jy, float jz, float far2) {
  float gx = fmaxf(fmaxf(lo.x - jx, jx - hi.x), 0.f);
  float gy = fmaxf(fmaxf(lo.y - jy, jy - hi.y), 0.f);
  float gz = fmaxf(fmaxf(lo.z - jz, jz - hi.z), 0.f);
  return gx * gx + gy * gy + gz * gz > far2;
}

// The pruning's f32 distance of a member at xm from a partner image at
// (jx, jy, jz) = frame + lattice shift: each difference, product and sum
// rounded once in this order (no contraction), so that a host restatement
// in f32 gets the same bits and the same inner lists.
__device__ __forceinline__ float nb_prune_r2(float4 xm, float jx, float jy, float jz) {
  float dx = __fsub_rn(xm.x, jx), dy = __fsub_rn(xm.y, jy), dz = __fsub_rn(xm.z, jz);
  return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

// The same pruning with a block of NB_PRUNE_WARPS warps per group: warp w
// takes the w-th contiguous share of the outer entries, stages what
// survives in shared memory, and the block writes the shares class by class
// (entries of more than NB_SPARSE_BITS members first, then by member count,
// each class in warp order), so the inner list holds the entries of the
// warp-per-group kernel, in a quarter of the dependent rounds, ordered for
// the pair kernel's sparse rounds.  A lane takes four entries a round, their loads and
// their partners' frames all issued before the first test, so a round costs
// two memory latencies for 128 entries.  Dynamic shared memory: list_cap
// entries.
//
// With `units`, each block also claims the units of its inner list from
// *unit_counter (zeroed by whoever decided the pruning) and writes them, so
// that no second launch scans the counts; the units then come in the order
// the blocks finish, which changes no force (each unit's work is the same)
// but the order of the per-unit energy partials: the deterministic mode keeps
// the scan.  Block 0 counts the pruning in *prunes.
#define NB_PRUNE_WARPS 4
// The pruning of group g by the calling block of NB_PRUNE_WARPS warps (every
// thread calls it, with the group's bounds already checked); returns the
// group's count of inner entries, the same in every thread.  Dynamic shared
// memory: list_cap entries (int2).
__device__ __forceinline__ int nb_prune_group(int64_t g, NbCell H, float rin2, int64_t list_cap,
                                              const int2 *__restrict__ slab, const int32_t *__restrict__ counts,
                                              const int32_t *__restrict__ order, const float4 *__restrict__ xq,
                                              int2 *__restrict__ slab_in, int32_t *__restrict__ counts_in,
                                              const double *__restrict__ x, double *__restrict__ x_prune,
                                              int32_t *unit_counter, int2 *__restrict__ units, int64_t units_cap,
                                              double *prunes) {
  extern __shared__ int2 s_stage[];
  // members m and m + 8 side by side for the packed tests: (x, x', y, y'), (z, z')
  __shared__ float4 s_mxy[NB_GROUP / 2];
  __shared__ float2 s_mz[NB_GROUP / 2];
  __shared__ int s_cls[NB_PRUNE_WARPS][NB_SPARSE_BITS + 1];
  __shared__ int s_unit0, s_nunits;
  __shared__ int2 s_qe[NB_PRUNE_WARPS][64];    // a warp's queue of entries that pass the box test
  __shared__ float4 s_qx[NB_PRUNE_WARPS][64];  // and their partners' images
  __shared__ unsigned s_live;
  __shared__ float3 s_lo, s_hi;
  const unsigned FULL = 0xffffffffu;
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (x_prune && threadIdx.x < 3 * NB_GROUP) {  // the positions of the pruning, for its test of validity
    int a = order[g * NB_GROUP + threadIdx.x / 3];
    if (a >= 0) x_prune[3 * a + threadIdx.x % 3] = x[3 * a + threadIdx.x % 3];
  }
  if (warp == 0) {
    float4 xme = xq[g * NB_GROUP + (lane & 15)];
    float ox = __shfl_sync(FULL, xme.x, lane + 8), oy = __shfl_sync(FULL, xme.y, lane + 8);
    float oz = __shfl_sync(FULL, xme.z, lane + 8);
    if (lane < NB_GROUP / 2) {
      s_mxy[lane] = make_float4(xme.x, ox, xme.y, oy);
      s_mz[lane] = make_float2(xme.z, oz);
    }
    bool on = lane < NB_GROUP && order[g * NB_GROUP + (lane & 15)] >= 0;
    unsigned live = __ballot_sync(FULL, on) & 0xffffu;
    float3 blo, bhi;
    nb_live_box(xme, on, blo, bhi);
    if (lane == 0) {
      s_live = live;
      s_lo = blo;
      s_hi = bhi;
    }
  }
  __syncthreads();
  unsigned live = s_live;
  const float3 box_lo = s_lo, box_hi = s_hi;
  const float far2 = rin2 * 1.0001f;
  int cnt = (int)min((int64_t)counts[g], list_cap);
  int share = ((cnt + NB_PRUNE_WARPS - 1) / NB_PRUNE_WARPS + 127) / 128 * 128;
  int lo = min(cnt, warp * share), hi = min(cnt, lo + share);
  int2 *stage = s_stage + lo;  // a warp's survivors never outnumber its share
  const int2 *src = slab + g * list_cap;
  int2 *qe = s_qe[warp];
  float4 *qx = s_qx[warp];
  int out = 0, qn = 0;  // survivors staged; entries queued (warp-uniform)
  // The member tests of the first `take` queued entries, a lane each, in
  // queue order (the order of the outer list): no lane idles on an entry
  // that the box test dropped.
  auto drain = [&](int take) {
    __syncwarp();
    unsigned inner = 0;
    int2 en = make_int2(0, 0);
    if (lane < take) {
      en = qe[lane];
      float4 xj = qx[lane];
      unsigned mm = (unsigned)en.y & live;
      // members m and m + 8 at once in packed f32x2 arithmetic, with the
      // roundings of nb_prune_r2 (x - y is x + (-y) exactly; products and
      // sums rounded once, in its order), so the bits are the same
      const float2 nx = make_float2(-xj.x, -xj.x), ny = make_float2(-xj.y, -xj.y), nz = make_float2(-xj.z, -xj.z);
#pragma unroll
      for (int m = 0; m < NB_GROUP / 2; ++m) {
        const float4 a = s_mxy[m];
        const float2 dx = __fadd2_rn(make_float2(a.x, a.y), nx), dy = __fadd2_rn(make_float2(a.z, a.w), ny);
        const float2 dz = __fadd2_rn(s_mz[m], nz);
        const float2 r2 = __fadd2_rn(__fadd2_rn(__fmul2_rn(dx, dx), __fmul2_rn(dy, dy)), __fmul2_rn(dz, dz));
        if (((mm >> m) & 1u) && r2.x <= rin2) inner |= 1u << m;
        if (((mm >> (m + 8)) & 1u) && r2.y <= rin2) inner |= 1u << (m + 8);
      }
    }
    unsigned has = __ballot_sync(FULL, inner != 0);
    if (inner)
      stage[out + __popc(has & ((1u << lane) - 1))] = make_int2(en.x, (int)(inner | ((unsigned)en.y & 0xffff0000u)));
    out += __popc(has);
    // the rest of the queue to its front
    __syncwarp();
    int2 re = make_int2(0, 0);
    float4 rx = make_float4(0.f, 0.f, 0.f, 0.f);
    bool move = take + lane < qn;
    if (move) {
      re = qe[take + lane];
      rx = qx[take + lane];
    }
    __syncwarp();
    if (move) {
      qe[lane] = re;
      qx[lane] = rx;
    }
    qn -= take;
  };
  for (int base = lo; base < hi; base += 128) {
    int2 en[4];
    float4 xj[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) en[j] = base + 32 * j + lane < hi ? src[base + 32 * j + lane] : make_int2(0, 0);
#pragma unroll
    for (int j = 0; j < 4; ++j) xj[j] = base + 32 * j + lane < hi ? xq[en[j].x] : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      bool pass = false;
      float jx = 0.f, jy = 0.f, jz = 0.f;
      if (base + 32 * j + lane < hi && ((unsigned)en[j].y & live & 0xffffu)) {
        int sx, sy, sz;
        nb_decode_image(((unsigned)en[j].y >> 16) & NB_IMAGE_BITS, sx, sy, sz);
        float3 t = nb_lattice_shift(sx, sy, sz, H);
        jx = __fadd_rn(xj[j].x, t.x);
        jy = __fadd_rn(xj[j].y, t.y);
        jz = __fadd_rn(xj[j].z, t.z);
        pass = !nb_beyond_box(box_lo, box_hi, jx, jy, jz, far2);
      }
      unsigned pb = __ballot_sync(FULL, pass);
      if (pass) {
        int at = qn + __popc(pb & ((1u << lane) - 1));
        qe[at] = en[j];
        qx[at] = make_float4(jx, jy, jz, 0.f);
      }
      qn += __popc(pb);
      if (qn >= 32) drain(32);
    }
  }
  if (qn > 0) drain(qn);
  // The inner list in classes by member count (class 0: more than
  // NB_SPARSE_BITS members, class c: c members), class by class, each class
  // in warp order and within a warp in the order staged.
  constexpr int NC = NB_SPARSE_BITS + 1;
  auto entry_class = [](int2 e) {
    int pc = __popc((unsigned)e.y & 0xffffu);
    return pc > NB_SPARSE_BITS ? 0 : pc;
  };
  int mine[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) mine[c] = 0;
  for (int i0 = 0; i0 < out; i0 += 32) {
    int cls = i0 + lane < out ? entry_class(stage[i0 + lane]) : -1;
#pragma unroll
    for (int c = 0; c < NC; ++c) mine[c] += __popc(__ballot_sync(FULL, cls == c));
  }
  if (lane == 0) {
#pragma unroll
    for (int c = 0; c < NC; ++c) s_cls[warp][c] = mine[c];
  }
  __syncthreads();
  int start[NC];
  int total = 0;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    int before = 0, all = 0;
    for (int w = 0; w < NB_PRUNE_WARPS; ++w) {
      int k = s_cls[w][c];
      if (w < warp) before += k;
      all += k;
    }
    start[c] = total + before;
    total += all;
  }
  for (int i0 = 0; i0 < out; i0 += 32) {
    int2 en = i0 + lane < out ? stage[i0 + lane] : make_int2(0, 0);
    int cls = i0 + lane < out ? entry_class(en) : -1;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      unsigned b = __ballot_sync(FULL, cls == c);
      if (cls == c) slab_in[g * list_cap + start[c] + __popc(b & ((1u << lane) - 1))] = en;
      start[c] += __popc(b);
    }
  }
  if (threadIdx.x == 0) {
    counts_in[g] = total;
    if (units) {
      int nu = (total + NB_UNIT - 1) / NB_UNIT;
      s_nunits = nu;
      s_unit0 = nu > 0 ? atomicAdd(unit_counter, nu) : 0;
      if (g == 0 && prunes) *prunes += 1.0;
    }
  }
  if (units) {
    __syncthreads();
    for (int k = threadIdx.x; k < s_nunits; k += blockDim.x)
      if (s_unit0 + k < units_cap) units[s_unit0 + k] = make_int2((int)g, k);
  }
  return total;
}

}  // namespace
