// The cluster-pair neighbor build on sm_100a.
//
// Replaces MDIR's emitted groups build (lib/Conversion/MDExecKernels/
// GroupsBuild.cpp: emitKeys 520, sortByKey 429, emitChunks 741, emitBoxes
// 912, emitLists 1098) behind the same contract (docs/neighbor-groups.md,
// Sections 1.1-1.3 and 4-5.2): every image of every non-excluded pair whose
// f32 distance is within the widened reach R' = R + 3e-6 (Lx+Ly+Lz) has
// exactly one bit, in the list of the group of the earlier place.
//
// The B200 design differs from the reference's: the cell sort is a counting
// sort into columns of about 16 atoms per column-width of height (so a
// group of 16 consecutive places of a column is close to a cube, with no
// sorting network); the search screens whole candidate groups against the
// group's bounding box, 32 candidates a ballot, then tests the 16 x 16
// pairs of two candidate groups per warp pass with the f32 test; the
// exclusion partners of the 16 members are sorted in shared memory and
// looked up by binary search; and the list of a group is a fixed slab of C
// entries (grown by the host when a build reports a longer list), so that
// the units of work come out in group order and every result is
// deterministic.
//
// Kernels (in launch order): nb_keys, scan, nb_scatter, nb_bin_sort,
// nb_col_groups, scan, nb_group_cols, nb_places, nb_boxes, nb_search,
// nb_unit_count, scan, nb_unit_write.
#include <cmath>
#include <cstdio>

#include "nb_context.h"
#include "nb_prune.cuh"
#include "nb_scan.cuh"

#define NB_EXCL_MAX 256

namespace {

// The brick of a cell: x + S H in [0, ax) x [0, by) x [0, cz), S found
// along c, then b, then a (with no tilts, per axis), each product and sum
// of f64 rounded as written.
__global__ void nb_keys(int64_t n, const double *__restrict__ x, double Lx, double Ly, double Lz,
                        double bx, double cx, double cy,
                        int Nx, int Ny, int Nz, float inv_wx, float inv_wy, float inv_hz,
                        int32_t *__restrict__ key, int32_t *__restrict__ bin_count,
                        float4 *__restrict__ atom_xw, char4 *__restrict__ atom_shift,
                        int32_t *__restrict__ sizes) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double v0 = x[3 * i], v1 = x[3 * i + 1], v2 = x[3 * i + 2];
  bool ok = isfinite(v0) && isfinite(v1) && isfinite(v2);
  double S0 = 0, S1 = 0, S2 = 0;
  double p0 = 0, p1 = 0, p2 = 0;
  if (ok) {
    S2 = -floor(v2 / Lz);
    p2 = __dadd_rn(v2, __dmul_rn(S2, Lz));
    p1 = __dadd_rn(v1, __dmul_rn(S2, cy));
    S1 = -floor(p1 / Ly);
    p1 = __dadd_rn(p1, __dmul_rn(S1, Ly));
    p0 = __dadd_rn(__dadd_rn(v0, __dmul_rn(S2, cx)), __dmul_rn(S1, bx));
    S0 = -floor(p0 / Lx);
    p0 = __dadd_rn(p0, __dmul_rn(S0, Lx));
    ok = fabs(S0) <= 100.0 && fabs(S1) <= 100.0 && fabs(S2) <= 100.0;
  }
  if (!ok) {
    key[i] = Nx * Ny * Nz;  // the bin of the positions that have no key
    atomicAdd(&bin_count[Nx * Ny * Nz], 1);
    atomicAdd(&sizes[NB_SIZE_NAN], 1);
    atom_xw[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    atom_shift[i] = make_char4(0, 0, 0, 0);
    return;
  }
  float w0 = (float)p0, w1 = (float)p1, w2 = (float)p2;
  int kx = min(max((int)(w0 * inv_wx), 0), Nx - 1);
  int ky = min(max((int)(w1 * inv_wy), 0), Ny - 1);
  int kz = min(max((int)(w2 * inv_hz), 0), Nz - 1);
  int k = (ky * Nx + kx) * Nz + kz;
  key[i] = k;
  atomicAdd(&bin_count[k], 1);
  atom_xw[i] = make_float4(w0, w1, w2, 1.f);
  atom_shift[i] = make_char4((signed char)S0, (signed char)S1, (signed char)S2, 0);
}

__global__ void nb_scatter(int64_t n, const int32_t *__restrict__ key,
                           const int32_t *__restrict__ bin_start, int32_t *__restrict__ bin_fill,
                           int32_t *__restrict__ sorted) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int k = key[i];
  int at = bin_start[k] + atomicAdd(&bin_fill[k], 1);
  sorted[at] = (int32_t)i;
}

// Each bin's atoms by number, so that the order does not depend on the
// threads (bins hold about half an atom on average).
__global__ void nb_bin_sort(int nbins, const int32_t *__restrict__ bin_start,
                            int32_t *__restrict__ sorted) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbins) return;
  int s = bin_start[b], e = bin_start[b + 1];
  for (int i = s + 1; i < e; ++i) {
    int v = sorted[i];
    int j = i - 1;
    while (j >= s && sorted[j] > v) {
      sorted[j + 1] = sorted[j];
      --j;
    }
    sorted[j + 1] = v;
  }
}

__global__ void nb_col_groups(int ncol, int Nz, const int32_t *__restrict__ bin_start,
                              int32_t *__restrict__ col_groups) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncol) return;
  int nc = bin_start[(c + 1) * Nz] - bin_start[c * Nz];
  col_groups[c] = (nc + NB_GROUP - 1) / NB_GROUP;
}

__global__ void nb_group_cols(int ncol, const int32_t *__restrict__ group_start, int64_t groups_cap,
                              int32_t *__restrict__ group_col, int32_t *__restrict__ sizes) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c == 0) {
    int g = group_start[ncol];
    sizes[NB_SIZE_GROUPS] = g;
    sizes[NB_SIZE_PLACES] = g * NB_GROUP;
    if (g > groups_cap) atomicOr(&sizes[NB_SIZE_OVERFLOW], 1);
  }
  if (c >= ncol) return;
  for (int g = group_start[c]; g < group_start[c + 1] && g < groups_cap; ++g) group_col[g] = c;
}

__global__ void nb_places(int nsorted_max, const int32_t *__restrict__ bin_start, int nvalid_bins,
                          const int32_t *__restrict__ sorted, const int32_t *__restrict__ key, int Nz,
                          const int32_t *__restrict__ group_start, int64_t places_cap,
                          const float4 *__restrict__ atom_xw, const char4 *__restrict__ atom_shift,
                          int32_t *__restrict__ order, int32_t *__restrict__ place_of,
                          char4 *__restrict__ shift, float4 *__restrict__ xw) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsorted_max) return;
  int nvalid = bin_start[nvalid_bins];
  int a = sorted[s];
  if (s >= nvalid) {  // positions with no key are in no group
    place_of[a] = -1;
    return;
  }
  int c = key[a] / Nz;
  int rank = s - bin_start[c * Nz];
  int64_t p = (int64_t)group_start[c] * NB_GROUP + rank;
  if (p >= places_cap) {
    place_of[a] = -1;
    return;
  }
  order[p] = a;
  place_of[a] = (int32_t)p;
  shift[p] = atom_shift[a];
  xw[p] = atom_xw[a];
}

__global__ void nb_boxes(int64_t groups_cap, const int32_t *__restrict__ sizes,
                         const int32_t *__restrict__ order, const float4 *__restrict__ xw,
                         float4 *__restrict__ box_lo, float4 *__restrict__ box_hi) {
  int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= groups_cap || g >= sizes[NB_SIZE_GROUPS]) return;
  float lo0 = INFINITY, lo1 = INFINITY, lo2 = INFINITY;
  float hi0 = -INFINITY, hi1 = -INFINITY, hi2 = -INFINITY;
  for (int u = 0; u < NB_GROUP; ++u) {
    int64_t p = g * NB_GROUP + u;
    if (order[p] < 0) continue;
    float4 v = xw[p];
    lo0 = fminf(lo0, v.x);
    lo1 = fminf(lo1, v.y);
    lo2 = fminf(lo2, v.z);
    hi0 = fmaxf(hi0, v.x);
    hi1 = fmaxf(hi1, v.y);
    hi2 = fmaxf(hi2, v.z);
  }
  box_lo[g] = make_float4(lo0, lo1, lo2, 0.f);
  box_hi[g] = make_float4(hi0, hi1, hi2, 0.f);
}

// The f32 distance of the pair test, the same for both orders of the pair:
// d = (x_B + s L) - x_A with A the atom of the smaller number and s the
// image of B relative to A; products and sums rounded one at a time.
__device__ __forceinline__ float nb_pair_r2(float4 xa, float4 xb, float sx, float sy, float sz) {
  float dx = __fsub_rn(__fadd_rn(xb.x, sx), xa.x);
  float dy = __fsub_rn(__fadd_rn(xb.y, sy), xa.y);
  float dz = __fsub_rn(__fadd_rn(xb.z, sz), xa.z);
  return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

struct SearchParams {
  float Lx, Ly, Lz;
  float bx, cx, cy;  // the tilts of a triclinic cell (tri != 0), else 0
  int tri;
  float wx, wy;
  int Nx, Ny;
  float R2f;     // (float)(R'^2)
  float Rbox;    // R' plus a margin, for the conservative box and window tests
  int64_t groups_cap;
  int64_t list_cap;
};

// W warps build the list of one group (W = 1: a warp a group, four groups
// a block; W = 4: a block a group).  Lanes 0-15 and 16-31 of a warp hold the
// members; a pass tests two candidate groups, one per half-warp, each lane
// one candidate place against the 16 members.  With W > 1 the columns of the
// window are cut into W contiguous shares, each warp stages its entries and
// the block writes them in warp order, so a list is the same for every W.
// The staging is shared memory (list_cap entries a warp) without `scratch`;
// with it, a ring of 64 entries a warp in shared memory whose full runs of
// 32 go to chunks claimed in the group's row of `scratch` (groups_cap x
// list_cap entries, the inner slab, which a build invalidates anyway), so
// that a block needs a few KB, not 4 list_cap x 8 B, and many blocks fit on
// an SM.
template <int W, bool BATCH>
__global__ void __launch_bounds__(128) nb_search_t(SearchParams P0, const NbFrameDev *__restrict__ frames,
                                                   const int32_t *__restrict__ group_frame,
                                                   const int32_t *sizes_in,
                                                   const int32_t *__restrict__ order,
                                                   const float4 *__restrict__ xw,
                                                   const float4 *__restrict__ box_lo,
                                                   const float4 *__restrict__ box_hi,
                                                   const int32_t *__restrict__ group_start,
                                                   const int32_t *__restrict__ excl_off,
                                                   const int32_t *__restrict__ excl,
                                                   int2 *__restrict__ slab, int32_t *__restrict__ counts,
                                                   int32_t *sizes, int2 *__restrict__ scratch) {
  constexpr int GPB = 4 / W;  // groups per block
  extern __shared__ int2 s_stage[];
  __shared__ int2 s_ring[W > 1 ? W : 1][64];
  __shared__ int s_fill;
  __shared__ int4 s_qi[4][64];    // a warp's queue: place, atom, image code, member bound | same group
  __shared__ float4 s_qx[4][64];  // and the place's frame
  __shared__ float4 s_mem[GPB][NB_GROUP];
  __shared__ int s_atom[GPB][NB_GROUP];
  __shared__ int s_key[GPB][NB_EXCL_MAX];
  __shared__ unsigned char s_ku[GPB][NB_EXCL_MAX];
  __shared__ int s_meta[GPB][4];  // nkeys, wide, kmin, kmax
  __shared__ int s_count[4];
  const unsigned FULL = 0xffffffffu;
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int u = lane & 15, half = lane >> 4;
  int gi = warp / W, part = warp % W;
  int64_t g = (int64_t)blockIdx.x * GPB + gi;
  int ngroups = sizes_in[NB_SIZE_GROUPS];
  bool live = g < ngroups && g < P0.groups_cap;
  if (W == 1 && !live) return;
  // a frame of a batch: its cell, grid, reach and first column
  SearchParams P = P0;
  int col0 = 0;
  if (BATCH && live) {
    const NbFrameDev &F = frames[group_frame[g]];
    P.Lx = F.Lf0;
    P.Ly = F.Lf1;
    P.Lz = F.Lf2;
    P.wx = F.wx;
    P.wy = F.wy;
    P.Nx = F.Nx;
    P.Ny = F.Ny;
    P.R2f = F.R2f;
    P.Rbox = F.Rbox;
    col0 = F.col0;
  }

  // members and the exclusion partners of the members: keys (partner atom,
  // member), sorted; by the first warp of the group
  if (live && part == 0) {
    int64_t pi = g * NB_GROUP + u;
    int ai = order[pi];
    float4 xi = xw[pi];
    if (half == 0) {
      xi.w = ai >= 0 ? 1.f : 0.f;
      s_mem[gi][u] = xi;
      s_atom[gi][u] = ai;
    }
    int rs = 0, re = 0;
    if (excl_off && half == 0 && ai >= 0) {
      rs = excl_off[ai];
      re = excl_off[ai + 1];
    }
    int cnt = re - rs;
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += y;
    }
    int nkeys = __shfl_sync(FULL, incl, 31);
    bool wide = nkeys > NB_EXCL_MAX;
    if (!wide) {
      int at = incl - cnt;
      for (int k = 0; k < cnt; ++k) {
        s_key[gi][at + k] = excl[rs + k];
        s_ku[gi][at + k] = (unsigned char)u;
      }
    } else if (lane == 0) {
      atomicAdd(&sizes[NB_SIZE_EXCL_WIDE], 1);
    }
    __syncwarp();
    int kmin = INT_MAX, kmax = INT_MIN;
    if (!wide && nkeys > 0) {
      // rank sort of the keys by (partner, member, position)
      int myk[NB_EXCL_MAX / 32];
      unsigned char myu[NB_EXCL_MAX / 32];
      int myr[NB_EXCL_MAX / 32];
      int mine = 0;
      for (int k = lane; k < nkeys; k += 32, ++mine) {
        int kv = s_key[gi][k];
        unsigned char ku = s_ku[gi][k];
        int r = 0;
        for (int t = 0; t < nkeys; ++t) {
          int tv = s_key[gi][t];
          r += (tv < kv) || (tv == kv && t < k);
        }
        myk[mine] = kv;
        myu[mine] = ku;
        myr[mine] = r;
        kmin = min(kmin, kv);
        kmax = max(kmax, kv);
      }
      __syncwarp();
      for (int m = 0; m < mine; ++m) {
        s_key[gi][myr[m]] = myk[m];
        s_ku[gi][myr[m]] = myu[m];
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        kmin = min(kmin, __shfl_xor_sync(FULL, kmin, o));
        kmax = max(kmax, __shfl_xor_sync(FULL, kmax, o));
      }
    }
    if (lane == 0) {
      s_meta[gi][0] = nkeys;
      s_meta[gi][1] = wide;
      s_meta[gi][2] = kmin;
      s_meta[gi][3] = kmax;
    }
    __syncwarp();
  }
  const bool chunked = W > 1 && scratch != nullptr;
  const int chunk_cap = (int)(P.list_cap / 32) + 1;  // chunk offsets a warp
  int *chunk_at = chunked ? (int *)s_stage + warp * chunk_cap : nullptr;
  int2 *ring = s_ring[W > 1 ? warp : 0];
  int rhead = 0, rn = 0, nchunks = 0;  // the ring's first entry and size; chunks written
  if (chunked && threadIdx.x == 0) s_fill = 0;
  if (W > 1) __syncthreads();
  else __syncwarp();
  int count = 0;
  int2 *stage = (W > 1 && !chunked) ? s_stage + (size_t)warp * P.list_cap : nullptr;
  if (live) {
    int nkeys = s_meta[gi][0];
    bool wide = s_meta[gi][1] != 0;
    int kmin = s_meta[gi][2], kmax = s_meta[gi][3];
    float4 lo = box_lo[g], hi = box_hi[g];
    NbCell H;
    H.ax = P.Lx;
    H.by = P.Ly;
    H.cz = P.Lz;
    H.bx = P.bx;
    H.cx = P.cx;
    H.cy = P.cy;
    float ci0 = 0.5f * (lo.x + hi.x), ci1 = 0.5f * (lo.y + hi.y), ci2 = 0.5f * (lo.z + hi.z);
    float wi0 = 0.5f * (hi.x - lo.x), wi1 = 0.5f * (hi.y - lo.y), wi2 = 0.5f * (hi.z - lo.z);
    int kx0 = (int)floorf((lo.x - P.Rbox) / P.wx), kx1 = (int)floorf((hi.x + P.Rbox) / P.wx);
    int ky0 = (int)floorf((lo.y - P.Rbox) / P.wy), ky1 = (int)floorf((hi.y + P.Rbox) / P.wy);
    int sz0 = (lo.z - P.Rbox < 0.f) ? -1 : 0;
    int sz1 = (hi.z + P.Rbox >= P.Lz) ? 1 : 0;
    float Rb2 = P.Rbox * P.Rbox;
    int nx = kx1 - kx0 + 1, nwin = (ky1 - ky0 + 1) * nx;
    int w0 = (int)((int64_t)nwin * part / W), w1 = (int)((int64_t)nwin * (part + 1) / W);

    // Places of the candidate groups that pass the test against this
    // group's box wait in a queue of 64 a warp; the member tests then run a
    // place a lane over 32 of them at once, in queue order (the order of the
    // window, so the list is the one of testing every place), and no lane
    // idles on a place that the box test dropped.
    int4 *qi = s_qi[warp];
    float4 *qx = s_qx[warp];
    int qh = 0, qn = 0;  // the queue's first entry and size (warp-uniform)
    auto drain = [&](int take) {
      __syncwarp();
      unsigned mask = 0;
      int pj = 0, code = 0;
      if (lane < take) {
        int4 e = qi[(qh + lane) & 63];
        float4 xj = qx[(qh + lane) & 63];
        pj = e.x;
        int aj = e.y;
        code = e.z;
        int uu = e.w & 15;
        bool same = ((e.w >> 4) & 1) != 0;
        int sx, sy, sz;
        nb_decode_image(code, sx, sy, sz);
        float3 t = nb_lattice_shift(sx, sy, sz, H);
        float fsx = t.x, fsy = t.y, fsz = t.z;
#pragma unroll 4
        for (int m = 0; m < NB_GROUP; ++m) {
          float4 xm = s_mem[gi][m];
          int am = s_atom[gi][m];
          // canonical orientation: A = smaller atom number
          bool jfirst = aj < am;
          float4 xa = jfirst ? xj : xm;
          float4 xb = jfirst ? xm : xj;
          float sgn = jfirst ? -1.f : 1.f;
          float r2 = nb_pair_r2(xa, xb, sgn * fsx, sgn * fsy, sgn * fsz);
          bool ok = (xm.w != 0.f) && (r2 <= P.R2f) && (!same || m < uu);
          mask |= ok ? (1u << m) : 0u;
        }
        if (mask) {
          if (!wide) {
            if (nkeys > 0 && aj >= kmin && aj <= kmax) {
              int lo_i = 0, hi_i = nkeys;
              while (lo_i < hi_i) {
                int mid = (lo_i + hi_i) >> 1;
                if (s_key[gi][mid] < aj) lo_i = mid + 1; else hi_i = mid;
              }
              for (int k = lo_i; k < nkeys && s_key[gi][k] == aj; ++k)
                mask &= ~(1u << s_ku[gi][k]);
            }
          } else {
            unsigned mm = mask;
            while (mm) {
              int m = __ffs(mm) - 1;
              mm &= mm - 1;
              int am = s_atom[gi][m];
              for (int k = excl_off[am]; k < excl_off[am + 1]; ++k)
                if (excl[k] == aj) mask &= ~(1u << m);
            }
          }
        }
      }
      unsigned has = __ballot_sync(FULL, mask != 0);
      if (chunked) {
        if (mask)
          ring[(rhead + rn + __popc(has & ((1u << lane) - 1))) & 63] =
              make_int2(pj, (int)(mask | ((unsigned)code << 16)));
        rn += __popc(has);
        if (rn >= 32) {  // a full run of 32 to a chunk of the group's scratch row
          __syncwarp();
          int claim = 0;
          if (lane == 0) claim = atomicAdd(&s_fill, 32);
          claim = __shfl_sync(FULL, claim, 0);
          if (claim + 32 <= P.list_cap) scratch[g * P.list_cap + claim + lane] = ring[(rhead + lane) & 63];
          if (lane == 0 && nchunks < chunk_cap) chunk_at[nchunks] = claim + 32 <= P.list_cap ? claim : -1;
          ++nchunks;
          rhead = (rhead + 32) & 63;
          rn -= 32;
          __syncwarp();
        }
      } else if (mask) {
        int at = count + __popc(has & ((1u << lane) - 1));
        int2 en = make_int2(pj, (int)(mask | ((unsigned)code << 16)));
        if (at < P.list_cap) {
          if (W > 1)
            stage[at] = en;
          else
            slab[g * P.list_cap + at] = en;
        }
      }
      count += __popc(has);
      qh = (qh + take) & 63;
      qn -= take;
      __syncwarp();
    };

    // The candidate groups of column c seen through the image T (code):
    // the box test, then the places that pass the test against this group's
    // box into the queue.
    auto visit = [&](int c, float fsx, float fsy, float fsz, int code) {
      int hb = max(group_start[c], (int)g), he = group_start[c + 1];
      for (int base = hb; base < he; base += 32) {
        int hc = base + lane;
        bool pass = false;
        if (hc < he) {
          float4 l2 = box_lo[hc], h2 = box_hi[hc];
          float d0 = fabsf(0.5f * (l2.x + h2.x) + fsx - ci0) - (wi0 + 0.5f * (h2.x - l2.x));
          float d1 = fabsf(0.5f * (l2.y + h2.y) + fsy - ci1) - (wi1 + 0.5f * (h2.y - l2.y));
          float d2 = fabsf(0.5f * (l2.z + h2.z) + fsz - ci2) - (wi2 + 0.5f * (h2.z - l2.z));
          d0 = fmaxf(d0, 0.f);
          d1 = fmaxf(d1, 0.f);
          d2 = fmaxf(d2, 0.f);
          pass = d0 * d0 + d1 * d1 + d2 * d2 <= Rb2;
        }
        unsigned bits = __ballot_sync(FULL, pass);
        while (bits) {
          int c0 = __ffs(bits) - 1;
          bits &= bits - 1;
          int c1 = -1;
          if (bits) {
            c1 = __ffs(bits) - 1;
            bits &= bits - 1;
          }
          int cand = half ? c1 : c0;
          bool keep = false;
          int pj = 0, aj = -1;
          float4 xj = make_float4(0.f, 0.f, 0.f, 0.f);
          bool same = false;
          if (cand >= 0) {
            int64_t h = base + cand;
            pj = (int)(h * NB_GROUP + u);
            aj = order[pj];
            if (aj >= 0) {
              xj = xw[pj];
              same = h == g;
              // the place against this group's box, with the margin of the window
              float xs = xj.x + fsx, ys = xj.y + fsy, zs = xj.z + fsz;
              float gx = fmaxf(fmaxf(lo.x - xs, xs - hi.x), 0.f);
              float gy = fmaxf(fmaxf(lo.y - ys, ys - hi.y), 0.f);
              float gz = fmaxf(fmaxf(lo.z - zs, zs - hi.z), 0.f);
              keep = gx * gx + gy * gy + gz * gz <= Rb2;
            }
          }
          unsigned kb = __ballot_sync(FULL, keep);
          if (keep) {
            int at = (qh + qn + __popc(kb & ((1u << lane) - 1))) & 63;
            qi[at] = make_int4(pj, aj, code, u | (same ? 16 : 0));
            qx[at] = xj;
          }
          qn += __popc(kb);
          if (qn >= 32) drain(32);
        }
      }
    };

    if (!P.tri) {
      // orthorhombic: the window of columns around the box, wrapped per axis
      for (int wi = w0; wi < w1; ++wi) {
        int ky = ky0 + wi / nx, kx = kx0 + wi % nx;
        int cy = ((ky % P.Ny) + P.Ny) % P.Ny;
        int sy = (ky - cy) / P.Ny;
        int cx = ((kx % P.Nx) + P.Nx) % P.Nx;
        int sx = (kx - cx) / P.Nx;
        int c = col0 + cy * P.Nx + cx;
        if (max(group_start[c], (int)g) >= group_start[c + 1]) continue;
        for (int sz = sz0; sz <= sz1; ++sz) {
          float3 t = nb_lattice_shift(sx, sy, sz, H);
          visit(c, t.x, t.y, t.z, nb_image_code(sx, sy, sz));
        }
      }
    } else {
      // triclinic: every lattice vector n that can bring a brick position
      // within the reach of the box (along c, then b, then a), each with the
      // brick's columns its window cuts; the (image, column) pairs are
      // shared among the W warps in this order.
      const float R = P.Rbox;
      auto each = [&](auto &&fn) {
        int nc0 = (int)floorf((lo.z - R) / H.cz), nc1 = (int)floorf((hi.z + R) / H.cz);
        for (int nc = nc0; nc <= nc1; ++nc) {
          float yc = (float)nc * H.cy, xc = (float)nc * H.cx;
          int nb0 = (int)floorf((lo.y - R - yc) / H.by), nb1 = (int)floorf((hi.y + R - yc) / H.by);
          for (int nb = nb0; nb <= nb1; ++nb) {
            float xb = xc + (float)nb * H.bx;
            int na0 = (int)floorf((lo.x - R - xb) / H.ax), na1 = (int)floorf((hi.x + R - xb) / H.ax);
            for (int na = na0; na <= na1; ++na) {
              float3 t = nb_lattice_shift(na, nb, nc, H);
              if (hi.z + R - t.z < 0.f || lo.z - R - t.z >= H.cz) continue;
              int ax0 = max(0, (int)floorf((lo.x - R - t.x) / P.wx));
              int ax1 = min(P.Nx - 1, (int)floorf((hi.x + R - t.x) / P.wx));
              int ay0 = max(0, (int)floorf((lo.y - R - t.y) / P.wy));
              int ay1 = min(P.Ny - 1, (int)floorf((hi.y + R - t.y) / P.wy));
              if (ax0 > ax1 || ay0 > ay1) continue;
              fn(na, nb, nc, t, ax0, ax1, ay0, ay1);
            }
          }
        }
      };
      int total = 0;
      each([&](int, int, int, float3, int ax0, int ax1, int ay0, int ay1) {
        total += (ax1 - ax0 + 1) * (ay1 - ay0 + 1);
      });
      int t0 = (int)((int64_t)total * part / W), t1 = (int)((int64_t)total * (part + 1) / W);
      int at = 0;
      each([&](int na, int nb, int nc, float3 t, int ax0, int ax1, int ay0, int ay1) {
        int nxw = ax1 - ax0 + 1, cnt = nxw * (ay1 - ay0 + 1);
        int lo_i = max(t0 - at, 0), hi_i = min(t1 - at, cnt);
        for (int k = lo_i; k < hi_i; ++k) {
          int c = col0 + (ay0 + k / nxw) * P.Nx + ax0 + k % nxw;
          if (max(group_start[c], (int)g) >= group_start[c + 1]) continue;
          visit(c, t.x, t.y, t.z, nb_image_code(na, nb, nc));
        }
        at += cnt;
      });
    }
    if (qn > 0) drain(qn);
  }
  if (W == 1) {
    if (lane == 0) {
      counts[g] = count;
      atomicMax(&sizes[NB_SIZE_LONGEST], count);
      if (count > P.list_cap) atomicOr(&sizes[NB_SIZE_OVERFLOW], 2);
    }
    return;
  }
  if (lane == 0) s_count[warp] = count;
  __syncthreads();
  if (!live) return;
  int at = 0, total = 0;
  for (int w = gi * W; w < gi * W + W; ++w) {
    if (w < warp) at += s_count[w];
    total += s_count[w];
  }
  if (chunked) {
    // this warp's chunks in the order written, then what its ring holds
    for (int k = 0; k < nchunks && k < chunk_cap; ++k) {
      int from = chunk_at[k];
      int to = at + 32 * k + lane;
      if (from >= 0 && to < P.list_cap) slab[g * P.list_cap + to] = scratch[g * P.list_cap + from + lane];
    }
    int to = at + 32 * nchunks + lane;
    if (lane < rn && to < P.list_cap) slab[g * P.list_cap + to] = ring[(rhead + lane) & 63];
  } else {
    int keep = (int)min((int64_t)count, P.list_cap);
    for (int i = lane; i < keep; i += 32)
      if (at + i < P.list_cap) slab[g * P.list_cap + at + i] = stage[i];
  }
  if (part == 0 && lane == 0) {
    counts[g] = total;
    atomicMax(&sizes[NB_SIZE_LONGEST], total);
    if (total > P.list_cap) atomicOr(&sizes[NB_SIZE_OVERFLOW], 2);
  }
}

__global__ void nb_unit_count(int64_t groups_cap, const int32_t *__restrict__ sizes,
                              const int32_t *__restrict__ counts, int64_t list_cap,
                              int32_t *__restrict__ unit_n) {
  int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= groups_cap) return;
  int c = 0;
  if (g < sizes[NB_SIZE_GROUPS]) c = (int)min((int64_t)counts[g], list_cap);
  unit_n[g] = (c + NB_UNIT - 1) / NB_UNIT;
}

__global__ void nb_unit_write(int64_t groups_cap, const int32_t *__restrict__ unit_n,
                              const int32_t *__restrict__ unit_start, int64_t units_cap,
                              int2 *__restrict__ units, int32_t *__restrict__ sizes) {
  int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g == 0) {
    int total = unit_start[groups_cap];
    sizes[NB_SIZE_UNITS] = total;
    if (total > units_cap) atomicOr(&sizes[NB_SIZE_OVERFLOW], 4);
  }
  if (g >= groups_cap) return;
  int s = unit_start[g];
  for (int k = 0; k < unit_n[g]; ++k)
    if (s + k < units_cap) units[s + k] = make_int2((int)g, k);
}

__global__ void nb_count_entries(int64_t groups_cap, const int32_t *sizes,
                                 const int32_t *__restrict__ counts, int32_t *out) {
  int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= groups_cap || g >= sizes[NB_SIZE_GROUPS]) return;
  atomicAdd(&out[NB_SIZE_ENTRIES], counts[g]);
}

// The pruning of the dual list (MDIR: emitGroupsPrune,
// lib/Conversion/MDExecToGPU/MDExecToGPU.cpp:9588; docs/neighbor-groups.md,
// Section 6.2): inner mask = outer mask and [r^2 <= R_in'^2] at the current
// frames, entries whose inner mask is empty dropped, the rest written in
// their order (a warp per group, ballot compaction), so that the inner list
// of a group is a deterministic function of the outer one and the frames.
__global__ void __launch_bounds__(128) nb_prune(int64_t groups_cap, const int32_t *__restrict__ sizes,
                                                NbCell H, float rin2, int64_t list_cap,
                                                const int2 *__restrict__ slab, const int32_t *__restrict__ counts,
                                                const int32_t *__restrict__ order, const float4 *__restrict__ xq,
                                                int2 *__restrict__ slab_in, int32_t *__restrict__ counts_in,
                                                const int *gate, const double *__restrict__ x,
                                                double *__restrict__ x_prune) {
  __shared__ float4 s_m[4][NB_GROUP];
  const unsigned FULL = 0xffffffffu;
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int64_t g = (int64_t)blockIdx.x * 4 + warp;
  if (gate && *gate == 0) return;
  if (g >= groups_cap || g >= sizes[NB_SIZE_GROUPS]) return;
  if (x_prune) {
    for (int k = lane; k < 3 * NB_GROUP; k += 32) {
      int a = order[g * NB_GROUP + k / 3];
      if (a >= 0) x_prune[3 * a + k % 3] = x[3 * a + k % 3];
    }
  }
  float4 xme = xq[g * NB_GROUP + (lane & 15)];
  if (lane < NB_GROUP) s_m[warp][lane] = xme;
  bool on = lane < NB_GROUP && order[g * NB_GROUP + (lane & 15)] >= 0;
  unsigned live = __ballot_sync(FULL, on) & 0xffffu;
  float3 box_lo, box_hi;
  nb_live_box(xme, on, box_lo, box_hi);
  const float far2 = rin2 * 1.0001f;
  __syncwarp();
  int cnt = (int)min((int64_t)counts[g], list_cap);
  int out = 0;
  for (int base = 0; base < cnt; base += 32) {
    int e = base + lane;
    unsigned inner = 0;
    int2 en = make_int2(0, 0);
    if (e < cnt) {
      en = slab[g * list_cap + e];
      unsigned mm = (unsigned)en.y & live & 0xffffu;
      int sx, sy, sz;
      nb_decode_image(((unsigned)en.y >> 16) & NB_IMAGE_BITS, sx, sy, sz);
      float4 xj = xq[en.x];
      float3 t = nb_lattice_shift(sx, sy, sz, H);
      float jx = __fadd_rn(xj.x, t.x), jy = __fadd_rn(xj.y, t.y), jz = __fadd_rn(xj.z, t.z);
      if (nb_beyond_box(box_lo, box_hi, jx, jy, jz, far2)) mm = 0;
      while (mm) {
        int m = __ffs(mm) - 1;
        mm &= mm - 1;
        float r2 = nb_prune_r2(s_m[warp][m], jx, jy, jz);
        if (r2 <= rin2) inner |= 1u << m;
      }
    }
    unsigned has = __ballot_sync(FULL, inner != 0);
    if (inner) {
      int at = out + __popc(has & ((1u << lane) - 1));
      slab_in[g * list_cap + at] = make_int2(en.x, (int)(inner | ((unsigned)en.y & 0xffff0000u)));
    }
    out += __popc(has);
  }
  if (lane == 0) counts_in[g] = out;
}

// 8 blocks an SM (64 registers, 8 bytes spilled) rather than the 7 that 66
// registers allowed: the 1,526 groups of the 23,550-atom box take 1.29 waves
// of blocks instead of 1.47 (the MD step 54.45 against 54.70 µs, side by side)
__global__ void __launch_bounds__(NB_PRUNE_WARPS * 32, 8)
    nb_prune_block(int64_t groups_cap, const int32_t *__restrict__ sizes, NbCell H, float rin2,
                   int64_t list_cap, const int2 *__restrict__ slab, const int32_t *__restrict__ counts,
                   const int32_t *__restrict__ order, const float4 *__restrict__ xq, int2 *__restrict__ slab_in,
                   int32_t *__restrict__ counts_in, const int *gate, const double *__restrict__ x,
                   double *__restrict__ x_prune, int32_t *unit_counter, int2 *__restrict__ units,
                   int64_t units_cap, double *prunes) {
  int64_t g = blockIdx.x;
  nb_grid_wait();  // the gate and the frames of the kernels before (a chained launch)
  if (gate && *gate == 0) return;  // no pruning due (decided on the device)
  if (g >= groups_cap || g >= sizes[NB_SIZE_GROUPS]) return;
  nb_prune_group(g, H, rin2, list_cap, slab, counts, order, xq, slab_in, counts_in, x, x_prune, unit_counter, units,
                 units_cap, prunes);
}

inline int blocks_for(int64_t n, int t) { return (int)((n + t - 1) / t > 0 ? (n + t - 1) / t : 1); }

}  // namespace

// Grid of the counting sort: columns of about 16 atoms per column-width of
// height, z bins of about half an atom.
static NbGrid nb_plan_grid(int64_t n, const double box[3]) {
  NbGrid G;
  double V = box[0] * box[1] * box[2];
  double rho = (n > 0 ? (double)n : 1.0) / V;
  double dcol = cbrt((double)NB_GROUP / rho);
  G.Nx = (int)std::min(256.0, std::max(1.0, std::floor(box[0] / dcol)));
  G.Ny = (int)std::min(256.0, std::max(1.0, std::floor(box[1] / dcol)));
  int64_t nz = 2 * n / (G.Nx * G.Ny);
  G.Nz = (int)std::max<int64_t>(1, std::min<int64_t>(nz, 1 << 20));
  G.wx = (float)(box[0] / G.Nx);
  G.wy = (float)(box[1] / G.Ny);
  G.hz = (float)(box[2] / G.Nz);
  return G;
}

#define NB_CHECK(x)                                                  \
  do {                                                               \
    cudaError_t e_ = (x);                                            \
    if (e_ != cudaSuccess) {                                         \
      fprintf(stderr, "mdrt_nb: %s: %s\n", #x, cudaGetErrorString(e_)); \
      return -1;                                                     \
    }                                                                \
  } while (0)

template <typename T>
static int nb_realloc(T *&p, int64_t count) {
  if (p) cudaFree(p);
  p = nullptr;
  if (count <= 0) count = 1;
  cudaError_t e = cudaMalloc((void **)&p, sizeof(T) * (size_t)count);
  return e == cudaSuccess ? 0 : -1;
}

// Sizes the buffers for n atoms, the planned columns and bins
// (c.plan_cols, c.plan_bins) and the list capacity C.
static int nb_reserve(NbCtx &c, int64_t list_cap) {
  int64_t n = c.n;
  int64_t cols = c.plan_cols;
  int64_t groups = (n + NB_GROUP - 1) / NB_GROUP + cols;  // at most one partial group a column
  int64_t bins = c.plan_bins + 1;
  if (bins > c.bins_cap) {
    int64_t cap = bins + bins / 4;
    if (nb_realloc(c.bin_count, cap) || nb_realloc(c.bin_start, cap + 1) || nb_realloc(c.bin_fill, cap))
      return -1;
    int64_t scr = cap / NB_SCAN_TILE + 8;
    int64_t scr2 = (groups + groups / 4) / NB_SCAN_TILE + 8;
    if (nb_realloc(c.scan_scratch, std::max(scr, std::max<int64_t>(scr2, 64)) + 4096)) return -1;
    c.bins_cap = cap;
  }
  if (cols + 1 > c.cols_cap) {
    int64_t cap = cols + cols / 4 + 1;
    if (nb_realloc(c.col_groups, cap) || nb_realloc(c.group_start, cap + 1)) return -1;
    c.cols_cap = cap;
  }
  bool regroup = groups > c.groups_cap;
  if (regroup) {
    int64_t cap = groups + groups / 4 + 16;
    if (nb_realloc(c.order, cap * NB_GROUP) || nb_realloc(c.shift, cap * NB_GROUP) ||
        nb_realloc(c.xw, cap * NB_GROUP) || nb_realloc(c.box_lo, cap) || nb_realloc(c.box_hi, cap) ||
        nb_realloc(c.group_col, cap) || nb_realloc(c.counts, cap) || nb_realloc(c.unit_n, cap) ||
        nb_realloc(c.unit_start, cap + 1) || nb_realloc(c.xq, cap * NB_GROUP) ||
        nb_realloc(c.xq_lo, cap * NB_GROUP) ||
        nb_realloc(c.typ_p, cap * NB_GROUP) || nb_realloc(c.acc, cap * NB_GROUP) ||
        nb_realloc(c.acc_fixed, cap * NB_GROUP * 3))
      return -1;
    if (c.pme.on) {
      if (nb_realloc(c.pme.pme_force, cap * NB_GROUP * 4) || nb_realloc(c.pme.potential, cap * NB_GROUP) ||
          nb_realloc(c.pme.tile_bin, cap * NB_GROUP) || nb_realloc(c.pme.tile_rank, cap * NB_GROUP) ||
          nb_realloc(c.pme.tile_sorted, cap * NB_GROUP))
        return -1;
    }
    NB_CHECK(cudaMemset(c.acc, 0, sizeof(float4) * cap * NB_GROUP));
    NB_CHECK(cudaMemset(c.acc_fixed, 0, sizeof(unsigned long long) * cap * NB_GROUP * 3));
    c.groups_cap = cap;
    c.places_cap = cap * NB_GROUP;
  }
  if (regroup || list_cap != c.list_cap) {
    if (nb_realloc(c.slab, c.groups_cap * list_cap)) return -1;
    c.list_cap = list_cap;
    int64_t units = c.groups_cap * ((list_cap + NB_UNIT - 1) / NB_UNIT);
    if (units > c.units_cap) {
      if (nb_realloc(c.units, units) || nb_realloc(c.unit_partials, units * 8)) return -1;
      c.units_cap = units;
    }
  }
  return 0;
}

static int64_t nb_initial_list_cap(int64_t n, const double box[3], double reach, const NbGrid &G) {
  double V = box[0] * box[1] * box[2];
  double rho = n / V;
  double R = reach + 3e-6 * (box[0] + box[1] + box[2]);
  double hz = NB_GROUP / (rho * G.wx * G.wy);
  double w0 = 0.5 * G.wx, w1 = 0.5 * G.wy, w2 = 0.5 * hz;
  double VR = 8 * w0 * w1 * w2 + 8 * (w0 * w1 + w1 * w2 + w2 * w0) * R +
              2 * M_PI * (w0 + w1 + w2) * R * R + 4.0 / 3.0 * M_PI * R * R * R;
  double est = 0.5 * rho * VR * 1.6 + 64;
  est = std::min(est, (double)n * 27.0 + 64);
  return ((int64_t)est + NB_UNIT - 1) / NB_UNIT * NB_UNIT;
}

// Lets `kernel` take `bytes` of dynamic shared memory on the current device
// beside its static shared memory (the default cap is 48 KB for both
// together); once per device and size.
#define NB_MAX_DEVICES 64
template <typename K>
static void nb_allow_smem(K kernel, size_t bytes, size_t (&configured)[NB_MAX_DEVICES]) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (bytes > 16 * 1024 && dev >= 0 && dev < NB_MAX_DEVICES && configured[dev] < bytes) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    configured[dev] = bytes;
  }
}

// Launches one build on `s`. Returns 0; the sizes are left in c.sizes (device).
static void nb_build_launch(NbCtx &c, const double *x, const double box[3], cudaStream_t s) {
  const NbGrid &G = c.grid;
  int64_t n = c.n;
  int nbins = G.nbins();
  cudaMemsetAsync(c.sizes, 0, sizeof(int32_t) * NB_SIZE_COUNT, s);
  cudaMemsetAsync(c.bin_count, 0, sizeof(int32_t) * (nbins + 1), s);
  cudaMemsetAsync(c.bin_fill, 0, sizeof(int32_t) * (nbins + 1), s);
  cudaMemsetAsync(c.order, 0xff, sizeof(int32_t) * c.places_cap, s);
  nb_keys<<<blocks_for(n, 256), 256, 0, s>>>(n, x, box[0], box[1], box[2], c.tilt[0], c.tilt[1], c.tilt[2],
                                            G.Nx, G.Ny, G.Nz,
                                            1.0f / G.wx, 1.0f / G.wy, 1.0f / G.hz, c.key,
                                            c.bin_count, c.atom_xw, c.atom_shift, c.sizes);
  nb_scan(c.bin_count, c.bin_start, nbins + 1, nullptr, c.scan_scratch, s);
  nb_scatter<<<blocks_for(n, 256), 256, 0, s>>>(n, c.key, c.bin_start, c.bin_fill, c.sorted);
  nb_bin_sort<<<blocks_for(nbins + 1, 256), 256, 0, s>>>(nbins + 1, c.bin_start, c.sorted);
  nb_col_groups<<<blocks_for(G.ncol(), 256), 256, 0, s>>>(G.ncol(), G.Nz, c.bin_start, c.col_groups);
  nb_scan(c.col_groups, c.group_start, G.ncol(), nullptr, c.scan_scratch, s);
  nb_group_cols<<<blocks_for(G.ncol(), 256), 256, 0, s>>>(G.ncol(), c.group_start, c.groups_cap,
                                                         c.group_col, c.sizes);
  nb_places<<<blocks_for(n, 256), 256, 0, s>>>((int)n, c.bin_start, nbins, c.sorted, c.key, G.Nz,
                                              c.group_start, c.places_cap, c.atom_xw, c.atom_shift,
                                              c.order, c.place_of, c.shift, c.xw);
  nb_boxes<<<blocks_for(c.groups_cap, 128), 128, 0, s>>>(c.groups_cap, c.sizes, c.order, c.xw,
                                                        c.box_lo, c.box_hi);
  SearchParams P;
  P.Lx = (float)box[0];
  P.Ly = (float)box[1];
  P.Lz = (float)box[2];
  P.bx = (float)c.tilt[0];
  P.cx = (float)c.tilt[1];
  P.cy = (float)c.tilt[2];
  P.tri = nb_triclinic(c) ? 1 : 0;
  P.wx = G.wx;
  P.wy = G.wy;
  P.Nx = G.Nx;
  P.Ny = G.Ny;
  // the widening: 3e-6 of the sum of the diagonal and the tilts' magnitudes
  double span = box[0] + box[1] + box[2] + fabs(c.tilt[0]) + fabs(c.tilt[1]) + fabs(c.tilt[2]);
  double Rw = c.reach + 3e-6 * span;
  P.R2f = (float)(Rw * Rw);
  P.Rbox = (float)(Rw + 2e-5 * span + 1e-6);
  P.groups_cap = c.groups_cap;
  P.list_cap = c.list_cap;
  // four warps a group staging in chunks of the inner slab when it is there
  // (a dual list), else in shared memory when that fits, else one warp
  bool chunked = c.slab_in && c.slab_in_entries >= c.groups_cap * c.list_cap;
  size_t stage = chunked ? sizeof(int) * 4 * (size_t)(c.list_cap / 32 + 1) : sizeof(int2) * 4 * (size_t)c.list_cap;
  if (stage <= 200 * 1024) {
    static size_t configured[NB_MAX_DEVICES] = {};
    nb_allow_smem(nb_search_t<4, false>, stage, configured);
    nb_search_t<4, false><<<(int)c.groups_cap, 128, stage, s>>>(P, nullptr, nullptr, c.sizes, c.order, c.xw,
                                                                c.box_lo, c.box_hi, c.group_start, c.excl_off,
                                                                c.excl, c.slab, c.counts, c.sizes,
                                                                chunked ? c.slab_in : nullptr);
  } else {
    nb_search_t<1, false><<<blocks_for(c.groups_cap, 4), 128, 0, s>>>(P, nullptr, nullptr, c.sizes, c.order, c.xw,
                                                                      c.box_lo, c.box_hi, c.group_start,
                                                                      c.excl_off, c.excl, c.slab, c.counts,
                                                                      c.sizes, nullptr);
  }
  nb_unit_count<<<blocks_for(c.groups_cap, 256), 256, 0, s>>>(c.groups_cap, c.sizes, c.counts,
                                                             c.list_cap, c.unit_n);
  nb_scan(c.unit_n, c.unit_start, (int)c.groups_cap, nullptr, c.scan_scratch, s);
  nb_unit_write<<<blocks_for(c.groups_cap, 256), 256, 0, s>>>(c.groups_cap, c.unit_n, c.unit_start,
                                                             c.units_cap, c.units, c.sizes);
  nb_count_entries<<<blocks_for(c.groups_cap, 256), 256, 0, s>>>(c.groups_cap, c.sizes, c.counts,
                                                                c.sizes);
}

void nb_build_launch_public(NbCtx &c, const double *x, const double box[3], cudaStream_t s) {
  nb_build_launch(c, x, box, s);
}

int nb_reserve_inner(NbCtx &c) {
  // the inner buffers follow the outer capacities
  int64_t G = c.groups_cap, C = c.list_cap, U = c.units_cap;
  c.slab_in_entries = 0;
  if (nb_realloc(c.slab_in, G * C) || nb_realloc(c.counts_in, G) || nb_realloc(c.unit_n_in, G) ||
      nb_realloc(c.unit_start_in, G + 1) || nb_realloc(c.units_in, U))
    return -1;
  c.slab_in_entries = G * C;
  if (!c.sizes_in) {
    if (cudaMalloc(&c.sizes_in, sizeof(int32_t) * NB_SIZE_COUNT) != cudaSuccess) return -1;
  }
  cudaMemset(c.sizes_in, 0, sizeof(int32_t) * NB_SIZE_COUNT);
  c.inner_valid = false;
  return 0;
}

void nb_prune_run(NbCtx &c, const double box[3], cudaStream_t s) {
  double Rw = c.inner_reach + 3e-6 * (box[0] + box[1] + box[2] + fabs(c.tilt[0]) + fabs(c.tilt[1]) + fabs(c.tilt[2]));
  size_t stage = sizeof(int2) * (size_t)c.list_cap;
  if (stage <= 200 * 1024) {
    static size_t configured[NB_MAX_DEVICES] = {};
    nb_allow_smem(nb_prune_block, stage, configured);
    nb_prune_block<<<(int)c.groups_cap, NB_PRUNE_WARPS * 32, stage, s>>>(
        c.groups_cap, c.sizes, nb_cell(c, box), (float)(Rw * Rw), c.list_cap, c.slab,
        c.counts, c.order, c.xq, c.slab_in, c.counts_in, nullptr, nullptr, nullptr, nullptr, nullptr, 0, nullptr);
  } else {
    nb_prune<<<blocks_for(c.groups_cap, 4), 128, 0, s>>>(c.groups_cap, c.sizes, nb_cell(c, box),
                                                        (float)(Rw * Rw), c.list_cap, c.slab,
                                                        c.counts, c.order, c.xq, c.slab_in, c.counts_in, nullptr,
                                                        nullptr, nullptr);
  }
  nb_unit_count<<<blocks_for(c.groups_cap, 256), 256, 0, s>>>(c.groups_cap, c.sizes, c.counts_in, c.list_cap,
                                                             c.unit_n_in);
  nb_scan(c.unit_n_in, c.unit_start_in, (int)c.groups_cap, nullptr, c.scan_scratch, s);
  nb_unit_write<<<blocks_for(c.groups_cap, 256), 256, 0, s>>>(c.groups_cap, c.unit_n_in, c.unit_start_in,
                                                             c.units_cap, c.units_in, c.sizes_in);
}

namespace {

// The units of the lists in one block: a scan of the groups' unit counts,
// then the units (group, ordinal) in group order, the same as the
// three-kernel path; with a gate, nothing unless it is set.  Counts one
// more pruning in *prunes.
__global__ void __launch_bounds__(1024) nb_units_one_block(int64_t groups_cap, const int32_t *__restrict__ sizes,
                                                           const int32_t *__restrict__ counts, int64_t list_cap,
                                                           int64_t units_cap, int32_t *__restrict__ unit_start,
                                                           int2 *__restrict__ units, int32_t *__restrict__ sizes_out,
                                                           const int *gate, double *prunes) {
  __shared__ int s_part[1024];
  if (gate && *gate == 0) return;
  int G = (int)min((int64_t)sizes[NB_SIZE_GROUPS], groups_cap);
  int t = threadIdx.x;
  int per = (G + (int)blockDim.x - 1) / (int)blockDim.x;
  int g0 = min(G, t * per), g1 = min(G, g0 + per);
  int local = 0;
  for (int g = g0; g < g1; ++g) local += ((int)min((int64_t)counts[g], list_cap) + NB_UNIT - 1) / NB_UNIT;
  s_part[t] = local;
  __syncthreads();
  for (int o = 1; o < (int)blockDim.x; o <<= 1) {
    int y = t >= o ? s_part[t - o] : 0;
    __syncthreads();
    s_part[t] += y;
    __syncthreads();
  }
  int at = s_part[t] - local;
  for (int g = g0; g < g1; ++g) {
    int n = ((int)min((int64_t)counts[g], list_cap) + NB_UNIT - 1) / NB_UNIT;
    unit_start[g] = at;
    for (int k = 0; k < n; ++k)
      if (at + k < units_cap) units[at + k] = make_int2(g, k);
    at += n;
  }
  if (t == (int)blockDim.x - 1) {
    sizes_out[NB_SIZE_UNITS] = s_part[t];
    if (prunes) *prunes += 1.0;
  }
}

}  // namespace

void nb_prune_gated(NbCtx &c, const double box[3], const int *gate, const double *x, double *x_prune,
                    double *prunes, int32_t *unit_counter, cudaStream_t s) {
  double Rw = c.inner_reach + 3e-6 * (box[0] + box[1] + box[2] + fabs(c.tilt[0]) + fabs(c.tilt[1]) + fabs(c.tilt[2]));
  size_t stage = sizeof(int2) * (size_t)c.list_cap;
  if (stage <= 200 * 1024) {
    static size_t configured[NB_MAX_DEVICES] = {};
    nb_allow_smem(nb_prune_block, stage, configured);
    // outside the deterministic mode the blocks claim their units themselves
    // (the counter is zeroed by the update that asked for the pruning)
    bool claim = !c.deterministic && unit_counter;
    nb_launch_chained(nb_prune_block, dim3((int)c.groups_cap), dim3(NB_PRUNE_WARPS * 32), stage, s, c.groups_cap,
                      c.sizes, nb_cell(c, box), (float)(Rw * Rw), c.list_cap, c.slab,
                      c.counts, c.order, c.xq, c.slab_in, c.counts_in, gate, x, x_prune,
                      claim ? unit_counter : nullptr, claim ? c.units_in : nullptr, c.units_cap,
                      claim ? prunes : nullptr);
    if (claim) return;
  } else {
    nb_prune<<<blocks_for(c.groups_cap, 4), 128, 0, s>>>(c.groups_cap, c.sizes, nb_cell(c, box),
                                                        (float)(Rw * Rw), c.list_cap, c.slab,
                                                        c.counts, c.order, c.xq, c.slab_in, c.counts_in, gate, x,
                                                        x_prune);
  }
  nb_units_one_block<<<1, 1024, 0, s>>>(c.groups_cap, c.sizes, c.counts_in, c.list_cap, c.units_cap, c.unit_start_in,
                                       c.units_in, c.sizes_in, gate, prunes);
}

// One complete build with count-then-grow: the list capacity C grows to a
// quarter more than the longest list and the build runs again until every
// list fits (MDIR: mdrtGroupsGrow, runtime/mdrt_cuda.c:3185, and the build
// loop of lib/Conversion/MDExecToGPU/MDExecToGPU.cpp:10107-10175).
int nb_build_run(NbCtx &c, const double *x, const double box[3], cudaStream_t s) {
  NbGrid G = nb_plan_grid(c.n, box);
  int64_t cap = c.list_cap;
  if (cap == 0) cap = nb_initial_list_cap(c.n, box, c.reach, G);
  c.grid = G;
  c.plan_cols = G.ncol();
  c.plan_bins = G.nbins();
  if (!c.key) {
    if (nb_realloc(c.key, c.n) || nb_realloc(c.sorted, c.n) || nb_realloc(c.atom_xw, c.n) ||
        nb_realloc(c.atom_shift, c.n) || nb_realloc(c.place_of, c.n))
      return -1;
  }
  for (int attempt = 0; attempt < 8; ++attempt) {
    if (nb_reserve(c, cap)) return -1;
    nb_build_launch(c, x, box, s);
    NB_CHECK(cudaMemcpyAsync(c.h_sizes, c.sizes, sizeof(int32_t) * NB_SIZE_COUNT,
                             cudaMemcpyDeviceToHost, s));
    NB_CHECK(cudaStreamSynchronize(s));
    NB_CHECK(cudaGetLastError());
    if (c.h_sizes[NB_SIZE_OVERFLOW] == 0) {
      c.built = true;
      c.builds++;
      for (int k = 0; k < 3; ++k) c.box_built[k] = box[k];
      c.inner_valid = false;
      if (c.inner_reach > 0.0) {
        int64_t key = c.groups_cap * 1000003 + c.list_cap * 7 + c.units_cap;
        if (key != c.inner_key || !c.slab_in) {
          if (nb_reserve_inner(c)) return -1;
          c.inner_key = key;
        }
      }
      return 0;
    }
    int64_t longest = c.h_sizes[NB_SIZE_LONGEST];
    int64_t want = (longest + longest / 4 + NB_UNIT - 1) / NB_UNIT * NB_UNIT;
    cap = std::max(cap, want);
    c.grows++;
  }
  return -1;
}

namespace {

// Copies the entries of each list from a slab of old_cap entries a group to
// one of new_cap (a thread per entry of the old slab).
__global__ void nb_copy_lists(int64_t groups, const int32_t *__restrict__ sizes, int64_t old_cap, int64_t new_cap,
                              const int32_t *__restrict__ counts, const int2 *__restrict__ src,
                              int2 *__restrict__ dst) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t g = t / old_cap, e = t - g * old_cap;
  if (g >= groups || g >= sizes[NB_SIZE_GROUPS]) return;
  if (e >= min((int64_t)counts[g], old_cap)) return;
  dst[g * new_cap + e] = src[g * old_cap + e];
}

}  // namespace

int nb_grow_lists_keep(NbCtx &c, int64_t longest, cudaStream_t s) {
  int64_t want = (longest + longest / 4 + NB_UNIT - 1) / NB_UNIT * NB_UNIT;
  if (want <= c.list_cap || !c.built) return 0;
  int64_t G = c.groups_cap, C0 = c.list_cap;
  int64_t units = G * ((want + NB_UNIT - 1) / NB_UNIT);
  bool inner = c.slab_in != nullptr;
  int2 *slab = nullptr, *slab_in = nullptr, *units_new = nullptr, *units_in = nullptr;
  double *partials = nullptr;
  auto fail = [&]() {
    for (void *p : {(void *)slab, (void *)slab_in, (void *)units_new, (void *)units_in, (void *)partials})
      if (p) cudaFree(p);
    return -1;
  };
  if (cudaMalloc(&slab, sizeof(int2) * G * want) != cudaSuccess) return fail();
  if (inner && cudaMalloc(&slab_in, sizeof(int2) * G * want) != cudaSuccess) return fail();
  if (units > c.units_cap) {
    if (cudaMalloc(&units_new, sizeof(int2) * units) != cudaSuccess ||
        cudaMalloc(&partials, sizeof(double) * 8 * units) != cudaSuccess)
      return fail();
    if (inner && cudaMalloc(&units_in, sizeof(int2) * units) != cudaSuccess) return fail();
  }
  int blocks = blocks_for(G * C0, 256);
  nb_copy_lists<<<blocks, 256, 0, s>>>(G, c.sizes, C0, want, c.counts, c.slab, slab);
  if (inner) nb_copy_lists<<<blocks, 256, 0, s>>>(G, c.sizes, C0, want, c.counts_in, c.slab_in, slab_in);
  if (units_new) {
    cudaMemcpyAsync(units_new, c.units, sizeof(int2) * c.units_cap, cudaMemcpyDeviceToDevice, s);
    if (inner) cudaMemcpyAsync(units_in, c.units_in, sizeof(int2) * c.units_cap, cudaMemcpyDeviceToDevice, s);
  }
  NB_CHECK(cudaStreamSynchronize(s));
  NB_CHECK(cudaGetLastError());
  cudaFree(c.slab);
  c.slab = slab;
  if (inner) {
    cudaFree(c.slab_in);
    c.slab_in = slab_in;
    c.slab_in_entries = G * want;
  }
  if (units_new) {
    cudaFree(c.units);
    cudaFree(c.unit_partials);
    c.units = units_new;
    c.unit_partials = partials;
    if (inner) {
      cudaFree(c.units_in);
      c.units_in = units_in;
    }
    c.units_cap = units;
  }
  c.list_cap = want;
  c.inner_key = c.groups_cap * 1000003 + c.list_cap * 7 + c.units_cap;
  c.grows++;
  return 0;
}

int nb_grow_lists(NbCtx &c, int64_t longest) {
  int64_t want = (longest + longest / 4 + NB_UNIT - 1) / NB_UNIT * NB_UNIT;
  if (want <= c.list_cap) return 0;
  c.grows++;
  return nb_reserve(c, want);
}

// ---------------------------------------------------------------------------
// The build of a batch of frames (mdrtNbBatch).  The same stages as one
// system's, each one launch over all frames: the bins and columns of frame
// f start at F.bin0 and F.col0, so that the counting sort, the scans and
// the groups are those of one grid laid end to end, and the search of a
// group reads its frame's cell, grid and reach.

namespace {

__global__ void nb_batch_keys(int64_t n, const double *__restrict__ x, const int32_t *__restrict__ atom_frame,
                              const NbFrameDev *__restrict__ frames, int nbins, int32_t *__restrict__ key,
                              int32_t *__restrict__ atom_col, int32_t *__restrict__ bin_count,
                              float4 *__restrict__ atom_xw, char4 *__restrict__ atom_shift,
                              int32_t *__restrict__ sizes) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const NbFrameDev &F = frames[atom_frame[i]];
  double v0 = x[3 * i], v1 = x[3 * i + 1], v2 = x[3 * i + 2];
  bool ok = isfinite(v0) && isfinite(v1) && isfinite(v2);
  double S0 = 0, S1 = 0, S2 = 0;
  if (ok) {
    S0 = -floor(v0 / F.L0);
    S1 = -floor(v1 / F.L1);
    S2 = -floor(v2 / F.L2);
    ok = fabs(S0) <= 100.0 && fabs(S1) <= 100.0 && fabs(S2) <= 100.0;
  }
  if (!ok) {
    key[i] = nbins;
    atom_col[i] = -1;
    atomicAdd(&bin_count[nbins], 1);
    atomicAdd(&sizes[NB_SIZE_NAN], 1);
    atom_xw[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    atom_shift[i] = make_char4(0, 0, 0, 0);
    return;
  }
  float w0 = (float)(v0 + S0 * F.L0), w1 = (float)(v1 + S1 * F.L1), w2 = (float)(v2 + S2 * F.L2);
  int kx = min(max((int)(w0 * F.inv_wx), 0), F.Nx - 1);
  int ky = min(max((int)(w1 * F.inv_wy), 0), F.Ny - 1);
  int kz = min(max((int)(w2 * F.inv_hz), 0), F.Nz - 1);
  int col = ky * F.Nx + kx;
  int k = F.bin0 + col * F.Nz + kz;
  key[i] = k;
  atom_col[i] = F.col0 + col;
  atomicAdd(&bin_count[k], 1);
  atom_xw[i] = make_float4(w0, w1, w2, 1.f);
  atom_shift[i] = make_char4((signed char)S0, (signed char)S1, (signed char)S2, 0);
}

__global__ void nb_batch_col_groups(int ncol, const int32_t *__restrict__ col_frame,
                                    const NbFrameDev *__restrict__ frames, const int32_t *__restrict__ bin_start,
                                    int32_t *__restrict__ col_groups) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncol) return;
  const NbFrameDev &F = frames[col_frame[c]];
  int b0 = F.bin0 + (c - F.col0) * F.Nz;
  int nc = bin_start[b0 + F.Nz] - bin_start[b0];
  col_groups[c] = (nc + NB_GROUP - 1) / NB_GROUP;
}

__global__ void nb_batch_places(int nsorted_max, const int32_t *__restrict__ bin_start, int nvalid_bins,
                                const int32_t *__restrict__ sorted, const int32_t *__restrict__ atom_col,
                                const int32_t *__restrict__ col_frame, const NbFrameDev *__restrict__ frames,
                                const int32_t *__restrict__ group_start, int64_t places_cap,
                                const float4 *__restrict__ atom_xw, const char4 *__restrict__ atom_shift,
                                int32_t *__restrict__ order, int32_t *__restrict__ place_of,
                                char4 *__restrict__ shift, float4 *__restrict__ xw) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsorted_max) return;
  int nvalid = bin_start[nvalid_bins];
  int a = sorted[s];
  if (s >= nvalid) {
    place_of[a] = -1;
    return;
  }
  int c = atom_col[a];
  const NbFrameDev &F = frames[col_frame[c]];
  int rank = s - bin_start[F.bin0 + (c - F.col0) * F.Nz];
  int64_t p = (int64_t)group_start[c] * NB_GROUP + rank;
  if (p >= places_cap) {
    place_of[a] = -1;
    return;
  }
  order[p] = a;
  place_of[a] = (int32_t)p;
  shift[p] = atom_shift[a];
  xw[p] = atom_xw[a];
}

__global__ void nb_batch_group_frames(int64_t groups_cap, const int32_t *__restrict__ sizes,
                                      const int32_t *__restrict__ group_col, const int32_t *__restrict__ col_frame,
                                      const NbFrameDev *__restrict__ frames, int32_t *__restrict__ group_frame,
                                      float4 *__restrict__ group_L) {
  int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= groups_cap || g >= sizes[NB_SIZE_GROUPS]) return;
  int f = col_frame[group_col[g]];
  group_frame[g] = f;
  group_L[g] = make_float4(frames[f].Lf0, frames[f].Lf1, frames[f].Lf2, 0.f);
}

// The units of frame f: [frame_units[2f], frame_units[2f + 1]).
__global__ void nb_batch_frame_units(int nframes, const NbFrameDev *__restrict__ frames,
                                     const int32_t *__restrict__ group_start, const int32_t *__restrict__ unit_start,
                                     int32_t *__restrict__ frame_units) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nframes) return;
  const NbFrameDev &F = frames[f];
  int g0 = group_start[F.col0], g1 = group_start[F.col0 + F.ncol];
  frame_units[2 * f] = unit_start[g0];
  frame_units[2 * f + 1] = unit_start[g1];
}

}  // namespace

// The grids of the frames (host): columns and bins end to end, the widened
// reach of each cell; uploads the frames and the column -> frame map.
static int nb_batch_plan(mdrtNbBatch &b, int64_t *list_cap_hint) {
  NbCtx &c = b.nb->c;
  int64_t bins = 0, cols = 0, cap = 0;
  std::vector<int32_t> col_frame;
  for (int f = 0; f < b.frames; ++f) {
    NbFrameDev &F = b.h_frames[f];
    const double *L = &b.h_boxes[3 * f];
    int64_t nf = b.atom0[f + 1] - b.atom0[f];
    NbGrid G = nb_plan_grid(std::max<int64_t>(nf, 1), L);
    F.L0 = L[0];
    F.L1 = L[1];
    F.L2 = L[2];
    F.Lf0 = (float)L[0];
    F.Lf1 = (float)L[1];
    F.Lf2 = (float)L[2];
    F.Nx = G.Nx;
    F.Ny = G.Ny;
    F.Nz = G.Nz;
    F.wx = G.wx;
    F.wy = G.wy;
    F.inv_wx = 1.0f / G.wx;
    F.inv_wy = 1.0f / G.wy;
    F.inv_hz = 1.0f / G.hz;
    F.bin0 = (int)bins;
    F.col0 = (int)cols;
    F.ncol = G.ncol();
    F.atom0 = (int)b.atom0[f];
    F.natoms = (int)nf;
    double Rw = c.reach + 3e-6 * (L[0] + L[1] + L[2]);
    F.R2f = (float)(Rw * Rw);
    F.Rbox = (float)(Rw + 2e-5 * (L[0] + L[1] + L[2]) + 1e-6);
    F.pref = c.coulomb / (M_PI * L[0] * L[1] * L[2]);
    F.pi2_beta2 = c.beta > 0 ? M_PI * M_PI / (c.beta * c.beta) : 0.0;
    bins += G.nbins();
    cols += G.ncol();
    col_frame.insert(col_frame.end(), G.ncol(), f);
    cap = std::max(cap, nb_initial_list_cap(std::max<int64_t>(nf, 1), L, c.reach, G));
  }
  if (bins >= (1ll << 31) - 2 || cols >= (1ll << 31) - 2) return -1;
  c.plan_cols = cols;
  c.plan_bins = bins;
  if (list_cap_hint) *list_cap_hint = cap;
  if (!b.frames_dev && nb_realloc(b.frames_dev, b.frames)) return -1;
  NB_CHECK(cudaMemcpy(b.frames_dev, b.h_frames.data(), sizeof(NbFrameDev) * b.frames, cudaMemcpyHostToDevice));
  if (cols > b.cols_alloc) {
    if (nb_realloc(b.col_frame, cols)) return -1;
    b.cols_alloc = cols;
  }
  NB_CHECK(cudaMemcpy(b.col_frame, col_frame.data(), sizeof(int32_t) * cols, cudaMemcpyHostToDevice));
  return 0;
}

static void nb_batch_build_launch(mdrtNbBatch &b, const double *x, cudaStream_t s) {
  NbCtx &c = b.nb->c;
  int64_t n = c.n;
  int nbins = (int)c.plan_bins;
  int ncol = (int)c.plan_cols;
  cudaMemsetAsync(c.sizes, 0, sizeof(int32_t) * NB_SIZE_COUNT, s);
  cudaMemsetAsync(c.bin_count, 0, sizeof(int32_t) * (nbins + 1), s);
  cudaMemsetAsync(c.bin_fill, 0, sizeof(int32_t) * (nbins + 1), s);
  cudaMemsetAsync(c.order, 0xff, sizeof(int32_t) * c.places_cap, s);
  nb_batch_keys<<<blocks_for(n, 256), 256, 0, s>>>(n, x, b.atom_frame, b.frames_dev, nbins, c.key, b.atom_col,
                                                  c.bin_count, c.atom_xw, c.atom_shift, c.sizes);
  nb_scan(c.bin_count, c.bin_start, nbins + 1, nullptr, c.scan_scratch, s);
  nb_scatter<<<blocks_for(n, 256), 256, 0, s>>>(n, c.key, c.bin_start, c.bin_fill, c.sorted);
  nb_bin_sort<<<blocks_for(nbins + 1, 256), 256, 0, s>>>(nbins + 1, c.bin_start, c.sorted);
  nb_batch_col_groups<<<blocks_for(ncol, 256), 256, 0, s>>>(ncol, b.col_frame, b.frames_dev, c.bin_start,
                                                           c.col_groups);
  nb_scan(c.col_groups, c.group_start, ncol, nullptr, c.scan_scratch, s);
  nb_group_cols<<<blocks_for(ncol, 256), 256, 0, s>>>(ncol, c.group_start, c.groups_cap, c.group_col, c.sizes);
  nb_batch_places<<<blocks_for(n, 256), 256, 0, s>>>((int)n, c.bin_start, nbins, c.sorted, b.atom_col,
                                                    b.col_frame, b.frames_dev, c.group_start, c.places_cap,
                                                    c.atom_xw, c.atom_shift, c.order, c.place_of, c.shift, c.xw);
  nb_boxes<<<blocks_for(c.groups_cap, 128), 128, 0, s>>>(c.groups_cap, c.sizes, c.order, c.xw, c.box_lo,
                                                        c.box_hi);
  nb_batch_group_frames<<<blocks_for(c.groups_cap, 256), 256, 0, s>>>(c.groups_cap, c.sizes, c.group_col,
                                                                     b.col_frame, b.frames_dev, b.group_frame,
                                                                     b.group_L);
  SearchParams P = {};
  P.groups_cap = c.groups_cap;
  P.list_cap = c.list_cap;
  // four warps a group stage in chunks of the batch's scratch rows
  bool chunked = b.search_scratch && b.search_scratch_entries >= c.groups_cap * c.list_cap;
  size_t stage = chunked ? sizeof(int) * 4 * (size_t)(c.list_cap / 32 + 1) : sizeof(int2) * 4 * (size_t)c.list_cap;
  if (b.search_warps == 4 && stage <= 200 * 1024) {
    static size_t configured[NB_MAX_DEVICES] = {};
    nb_allow_smem(nb_search_t<4, true>, stage, configured);
    nb_search_t<4, true><<<(int)c.groups_cap, 128, stage, s>>>(P, b.frames_dev, b.group_frame, c.sizes, c.order,
                                                               c.xw, c.box_lo, c.box_hi, c.group_start, c.excl_off,
                                                               c.excl, c.slab, c.counts, c.sizes,
                                                               chunked ? b.search_scratch : nullptr);
  } else {
    nb_search_t<1, true><<<blocks_for(c.groups_cap, 4), 128, 0, s>>>(P, b.frames_dev, b.group_frame, c.sizes,
                                                                     c.order, c.xw, c.box_lo, c.box_hi,
                                                                     c.group_start, c.excl_off, c.excl, c.slab,
                                                                     c.counts, c.sizes, nullptr);
  }
  nb_unit_count<<<blocks_for(c.groups_cap, 256), 256, 0, s>>>(c.groups_cap, c.sizes, c.counts, c.list_cap,
                                                             c.unit_n);
  nb_scan(c.unit_n, c.unit_start, (int)c.groups_cap, nullptr, c.scan_scratch, s);
  nb_unit_write<<<blocks_for(c.groups_cap, 256), 256, 0, s>>>(c.groups_cap, c.unit_n, c.unit_start, c.units_cap,
                                                             c.units, c.sizes);
  nb_count_entries<<<blocks_for(c.groups_cap, 256), 256, 0, s>>>(c.groups_cap, c.sizes, c.counts, c.sizes);
  nb_batch_frame_units<<<blocks_for(b.frames, 128), 128, 0, s>>>(b.frames, b.frames_dev, c.group_start,
                                                                c.unit_start, b.frame_units);
}

int nb_batch_build_run(mdrtNbBatch &b, const double *x, cudaStream_t s) {
  NbCtx &c = b.nb->c;
  int64_t hint = 0;
  if (nb_batch_plan(b, &hint)) return -1;
  int64_t cap = std::max<int64_t>(c.list_cap, hint);
  if (!c.key) {
    if (nb_realloc(c.key, c.n) || nb_realloc(c.sorted, c.n) || nb_realloc(c.atom_xw, c.n) ||
        nb_realloc(c.atom_shift, c.n) || nb_realloc(c.place_of, c.n) || nb_realloc(b.atom_col, c.n))
      return -1;
  }
  if (!b.frame_units && nb_realloc(b.frame_units, 2 * (int64_t)b.frames)) return -1;
  for (int attempt = 0; attempt < 8; ++attempt) {
    if (nb_reserve(c, cap)) return -1;
    if (c.groups_cap > b.groups_alloc) {
      if (nb_realloc(b.group_frame, c.groups_cap) || nb_realloc(b.group_L, c.groups_cap)) return -1;
      b.groups_alloc = c.groups_cap;
    }
    if (b.search_warps == 4 && b.search_scratch_entries < c.groups_cap * c.list_cap) {
      b.search_scratch_entries = 0;
      if (nb_realloc(b.search_scratch, c.groups_cap * c.list_cap)) return -1;
      b.search_scratch_entries = c.groups_cap * c.list_cap;
    }
    nb_batch_build_launch(b, x, s);
    NB_CHECK(cudaMemcpyAsync(c.h_sizes, c.sizes, sizeof(int32_t) * NB_SIZE_COUNT, cudaMemcpyDeviceToHost, s));
    NB_CHECK(cudaStreamSynchronize(s));
    NB_CHECK(cudaGetLastError());
    if (c.h_sizes[NB_SIZE_OVERFLOW] == 0) {
      c.built = true;
      c.builds++;
      c.inner_valid = false;
      return 0;
    }
    int64_t longest = c.h_sizes[NB_SIZE_LONGEST];
    int64_t want = (longest + longest / 4 + NB_UNIT - 1) / NB_UNIT * NB_UNIT;
    cap = std::max(cap, want);
    c.grows++;
  }
  return -1;
}
