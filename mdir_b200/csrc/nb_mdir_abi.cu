// MDIR's own runtime names for the neighbor groups and the cuFFT transforms,
// with the memref descriptors of MLIR's C interface, so that a host program
// (or a patched MDIR emitter call site) that binds those names finds them in
// this library.
//
// The registry of groups follows runtime/mdrt_cuda.c:2994-3330 and the slot
// table of include/mdir/Runtime/GroupsABI.h:10-44 (ABI version 3):
//   - a handle (an int64) owns one device buffer of 32-bit values per slot,
//     sized by the slot's shape (places, groups = places / 16, entries =
//     64 blocks, blocks, ...); the outer list's slots (0-6) are allocated
//     with the handle, the others where first asked for;
//   - mdrtGroupsGrow makes room for more places or blocks, a quarter more
//     than asked, and drops what the buffers held (the caller builds again);
//   - mdrtGroupsBuilt returns the growths of the lists since the last
//     completed build and marks the structure built;
//   - mdrtGroupsReserveBlockOf sizes the block-of buffer;
//   - _mlir_ciface_mdrtGroupsBuffer / _mlir_ciface_mdrtGroupsPlaced return
//     a slot as a memref of rank 1, and the placed positions as one of rank
//     2 ([places, 3] f32).
// Where MDIR aborts (an invalid slot, a failed allocation), these entries
// print to stderr, return an empty descriptor, and leave the status for
// mdrtGroupsLastStatus.
//
// What fills the slots: this library's build (mdrtNbBuild) keeps its lists
// in its own context; mdrtNbGroupsExport copies them into a registry in
// MDIR's slot layout (order, counts, entries and masks in blocks of 64,
// the group and ordinal of each block, shifts, the pruned lists by blocks,
// the active blocks and their count, the placed positions).  The values are
// this library's: an entry's partner place, its mask of 16 members and the
// image code of include/mdrt_nb.h in bits 16-30 of the mask, the shifts as
// int8x4, the positions in the centred frames of the build.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>

#include <cufft.h>

#include "../../include/mdrt_nb.h"
#include "nb_context.h"

namespace {

// The length of slot `slot` in 32-bit values (GroupsABI.h's shapes).
enum Shape { PLACES, GROUPS, ENTRIES, BLOCKS, BLOCK_OF, SCALAR, RUNS, WIDE_RUNS, PLACED, SEGMENT_LISTS, SEGMENTS };
const Shape kShape[MDRT_GROUPS_BUFFERS] = {
    PLACES,  GROUPS, ENTRIES,  ENTRIES,   BLOCKS, BLOCKS, PLACES,        ENTRIES,       ENTRIES,      BLOCKS,
    BLOCK_OF, BLOCKS, SCALAR,  RUNS,      WIDE_RUNS, PLACED, SEGMENT_LISTS, SEGMENT_LISTS, PLACES, ENTRIES,
    ENTRIES, BLOCKS, BLOCKS,   SEGMENTS};

struct Groups {
  int device = 0;
  void *data[MDRT_GROUPS_BUFFERS] = {};
  int64_t places = 0, blocks = 0, block_of = 0;
  bool built = false;
  int64_t late_growths = 0;
  int64_t segments = 1;
};

int32_t g_last_status = MDRT_NB_OK;
std::mutex g_groups_mutex;

void note(int32_t status, const char *what) {
  std::lock_guard<std::mutex> lock(g_groups_mutex);
  g_last_status = status;
  if (what) fprintf(stderr, "mdrt_nb: %s\n", what);
}

int64_t length_of(const Groups &g, int slot) {
  switch (kShape[slot]) {
    case PLACES: return g.places;
    case GROUPS: return g.places / 16;
    case ENTRIES: return g.blocks * 64;
    case BLOCKS: return g.blocks;
    case BLOCK_OF: return g.block_of > 0 ? g.block_of : 1;
    case SCALAR: return 1;
    case RUNS: return g.blocks / 32 + 1;
    case WIDE_RUNS: return g.blocks / 1024 + 1;
    case PLACED: return g.places * 3;
    case SEGMENT_LISTS: return g.places / 16 * g.segments;
    case SEGMENTS: return g.segments + 1;
  }
  return 0;
}

bool allocate(Groups &g, int slot) {
  void *p = nullptr;
  size_t bytes = (size_t)length_of(g, slot) * sizeof(int32_t);
  if (cudaMalloc(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    note(MDRT_NB_CUDA_ERROR, "the groups registry could not allocate a buffer");
    return false;
  }
  g.data[slot] = p;
  return true;
}

void release(Groups &g) {
  for (int s = 0; s < MDRT_GROUPS_BUFFERS; ++s) {
    if (g.data[s]) cudaFree(g.data[s]);
    g.data[s] = nullptr;
  }
}

bool allocate_outer(Groups &g) {
  for (int s = 0; s < MDRT_GROUPS_INNER_ENTRIES; ++s)
    if (!allocate(g, s)) return false;
  return true;
}

Groups *from_handle(int64_t handle) { return reinterpret_cast<Groups *>((intptr_t)handle); }

// ---- export of a context's lists into MDIR's slots ------------------------

// Places: order, shifts (int8x4 as one 32-bit value) and the placed
// positions (three f32 a place).
__global__ void abi_places(int64_t places, const int32_t *__restrict__ order, const char4 *__restrict__ shift,
                           const float4 *__restrict__ xq, int32_t *__restrict__ o_order,
                           int32_t *__restrict__ o_shift, float *__restrict__ o_placed) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= places) return;
  o_order[p] = order[p];
  char4 s = shift[p];
  int32_t packed;
  memcpy(&packed, &s, sizeof(packed));
  o_shift[p] = packed;
  float4 v = xq[p];
  o_placed[3 * p] = v.x;
  o_placed[3 * p + 1] = v.y;
  o_placed[3 * p + 2] = v.z;
}

// Blocks: the 64 entries of unit b of a list, its group and ordinal, and
// (for the pruned lists) the entries the block holds.  Past a list's end an
// entry is -1 with mask 0.
__global__ void abi_blocks(int64_t nunits, const int2 *__restrict__ units, const int2 *__restrict__ slab,
                           const int32_t *__restrict__ counts, int64_t list_cap, int32_t *__restrict__ o_entries,
                           int32_t *__restrict__ o_masks, int32_t *__restrict__ o_groups,
                           int32_t *__restrict__ o_ordinals, int32_t *__restrict__ o_block_counts) {
  int64_t b = blockIdx.x;
  if (b >= nunits) return;
  int2 u = units[b];
  int cnt = (int)min((int64_t)counts[u.x], list_cap);
  int k = threadIdx.x;  // 64 threads
  int idx = u.y * 64 + k;
  int2 e = idx < cnt ? slab[(int64_t)u.x * list_cap + idx] : make_int2(-1, 0);
  o_entries[b * 64 + k] = e.x;
  o_masks[b * 64 + k] = e.y;
  if (k == 0) {
    if (o_groups) o_groups[b] = u.x;
    if (o_ordinals) o_ordinals[b] = u.y;
    if (o_block_counts) o_block_counts[b] = max(0, min(64, cnt - u.y * 64));
  }
}

__global__ void abi_copy_i32(int64_t n, const int32_t *__restrict__ in, int32_t *__restrict__ out) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[i];
}

__global__ void abi_iota(int64_t n, int32_t *__restrict__ out, int32_t *__restrict__ count) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (int32_t)i;
  if (i == 0) *count = (int32_t)n;
}

// ---- the Gaussian influence of the backward transform ---------------------

// complex[(x ky + y) (kz/2 + 1) + z] *= (tx[2 kx + x] ty[2 ky + y] tz[2 kz + z])
//                                      / (tx[kx + x] + ty[ky + y] + tz[kz + z]),
// 0 where the denominator is 0; the three rows of each axis k, in the
// order of the axes, are its wave numbers, their squares and its factors.
__global__ void abi_gaussian_scale(int64_t k1, int64_t k2, int64_t k3, const float *__restrict__ tables,
                                   float2 *__restrict__ spec) {
  int64_t h = k3 / 2 + 1;
  int64_t total = k1 * k2 * h;
  const float *tx = tables, *ty = tables + 3 * k1, *tz = ty + 3 * k2;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t z = i % h, row = i / h;
    int64_t y = row % k2, x = row / k2;
    float squared = (tx[k1 + x] + ty[k2 + y]) + tz[k3 + z];
    float product = (tx[2 * k1 + x] * ty[2 * k2 + y]) * tz[2 * k3 + z];
    float f = squared == 0.f ? 0.f : product * (1.0f / squared);
    float2 v = spec[i];
    spec[i] = make_float2(v.x * f, v.y * f);
  }
}

cudaStream_t g_abi_stream = nullptr;

}  // namespace

extern "C" {

int32_t mdrtGroupsLastStatus(void) {
  std::lock_guard<std::mutex> lock(g_groups_mutex);
  int32_t s = g_last_status;
  g_last_status = MDRT_NB_OK;
  return s;
}

int64_t mdrtGroupsCreate(int64_t places, int64_t blocks) {
  Groups *g = new (std::nothrow) Groups();
  if (!g) {
    note(MDRT_NB_INVALID_ARGUMENT, "out of host memory for a groups registry");
    return 0;
  }
  cudaGetDevice(&g->device);
  g->places = (places + 15) / 16 * 16;
  g->blocks = blocks > 0 ? blocks : 1;
  if (!allocate_outer(*g)) {
    release(*g);
    delete g;
    return 0;
  }
  return (int64_t)(intptr_t)g;
}

int32_t mdrtGroupsDestroy(int64_t handle) {
  Groups *g = from_handle(handle);
  if (!g) return MDRT_NB_INVALID_ARGUMENT;
  cudaDeviceSynchronize();
  release(*g);
  delete g;
  return MDRT_NB_OK;
}

void _mlir_ciface_mdrtGroupsBuffer(mdrtMemRef1D *result, int64_t handle, int64_t which) {
  if (!result) return;
  memset(result, 0, sizeof(*result));
  Groups *g = from_handle(handle);
  if (!g || which < 0 || which >= MDRT_GROUPS_BUFFERS) {
    char msg[96];
    snprintf(msg, sizeof msg, "invalid groups buffer slot %lld (expected 0..%d)", (long long)which,
             MDRT_GROUPS_BUFFERS - 1);
    note(MDRT_NB_INVALID_ARGUMENT, msg);
    return;
  }
  if (!g->data[which] && !allocate(*g, (int)which)) return;
  result->allocated = g->data[which];
  result->aligned = g->data[which];
  result->offset = 0;
  result->size = length_of(*g, (int)which);
  result->stride = 1;
}

void _mlir_ciface_mdrtGroupsPlaced(mdrtMemRef2D *result, int64_t handle) {
  if (!result) return;
  memset(result, 0, sizeof(*result));
  Groups *g = from_handle(handle);
  if (!g) {
    note(MDRT_NB_INVALID_ARGUMENT, "no groups registry");
    return;
  }
  if (!g->data[MDRT_GROUPS_PLACED] && !allocate(*g, MDRT_GROUPS_PLACED)) return;
  result->allocated = g->data[MDRT_GROUPS_PLACED];
  result->aligned = g->data[MDRT_GROUPS_PLACED];
  result->offset = 0;
  result->sizes[0] = g->places;
  result->sizes[1] = 3;
  result->strides[0] = 3;
  result->strides[1] = 1;
}

void mdrtGroupsGrow(int64_t handle, int64_t places, int64_t blocks) {
  Groups *g = from_handle(handle);
  if (!g) {
    note(MDRT_NB_INVALID_ARGUMENT, "no groups registry");
    return;
  }
  if (places <= g->places && blocks <= g->blocks) return;
  cudaDeviceSynchronize();  // no kernel may still use the buffers that are freed
  release(*g);
  if (places > g->places) g->places = (places + places / 4 + 15) / 16 * 16;
  bool lists = blocks > g->blocks;
  if (lists) g->blocks = blocks + blocks / 4;
  allocate_outer(*g);
  if (g->built && lists) ++g->late_growths;
}

int64_t mdrtGroupsBuilt(int64_t handle) {
  Groups *g = from_handle(handle);
  if (!g) {
    note(MDRT_NB_INVALID_ARGUMENT, "no groups registry");
    return 0;
  }
  int64_t late = g->late_growths;
  g->built = true;
  g->late_growths = 0;
  return late;
}

void mdrtGroupsReserveBlockOf(int64_t handle, int64_t length) {
  Groups *g = from_handle(handle);
  if (!g) {
    note(MDRT_NB_INVALID_ARGUMENT, "no groups registry");
    return;
  }
  if (length <= g->block_of && g->data[MDRT_GROUPS_BLOCK_OF]) return;
  if (length > g->block_of) g->block_of = length + length / 4;
  if (g->data[MDRT_GROUPS_BLOCK_OF]) {
    cudaDeviceSynchronize();
    cudaFree(g->data[MDRT_GROUPS_BLOCK_OF]);
    g->data[MDRT_GROUPS_BLOCK_OF] = nullptr;
  }
  allocate(*g, MDRT_GROUPS_BLOCK_OF);
}

int32_t mdrtNbGroupsExport(mdrtNb *ctx, int64_t handle, void *stream) {
  Groups *g = from_handle(handle);
  if (!ctx || !g) return MDRT_NB_INVALID_ARGUMENT;
  NbCtx &c = ctx->c;
  if (!c.built) return MDRT_NB_NOT_BUILT;
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t groups = c.h_sizes[NB_SIZE_GROUPS], places = 16 * groups;
  const int64_t units = std::min((int64_t)c.h_sizes[NB_SIZE_UNITS], c.units_cap);
  int32_t inner_units = 0;
  if (c.inner_valid && c.sizes_in) {
    if (cudaMemcpyAsync(&inner_units, c.sizes_in + NB_SIZE_UNITS, sizeof(int32_t), cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return MDRT_NB_CUDA_ERROR;
    inner_units = (int32_t)std::min((int64_t)inner_units, c.units_cap);
  }
  mdrtGroupsGrow(handle, places, std::max<int64_t>(units, inner_units));
  int want[] = {MDRT_GROUPS_PLACED, MDRT_GROUPS_INNER_ENTRIES, MDRT_GROUPS_INNER_MASKS,
                MDRT_GROUPS_INNER_COUNTS, MDRT_GROUPS_ACTIVE_UNITS, MDRT_GROUPS_ACTIVE_COUNT};
  for (int w : want)
    if (!g->data[w] && !allocate(*g, w)) return MDRT_NB_CUDA_ERROR;
  auto I = [&](int slot) { return (int32_t *)g->data[slot]; };
  if (places)
    abi_places<<<(unsigned)((places + 255) / 256), 256, 0, s>>>(places, c.order, c.shift, c.xq, I(0), I(6),
                                                                   (float *)g->data[MDRT_GROUPS_PLACED]);
  if (groups) abi_copy_i32<<<(unsigned)((groups + 255) / 256), 256, 0, s>>>(groups, c.counts, I(1));
  if (units)
    abi_blocks<<<(unsigned)units, 64, 0, s>>>(units, c.units, c.slab, c.counts, c.list_cap, I(2), I(3), I(4), I(5),
                                              nullptr);
  // the pruned lists by blocks, each with the entries it holds, and the
  // active blocks (every block of the pruned lists holds some)
  if (inner_units)
    abi_blocks<<<(unsigned)inner_units, 64, 0, s>>>(inner_units, c.units_in, c.slab_in, c.counts_in, c.list_cap,
                                                    I(7), I(8), nullptr, nullptr, I(9));
  abi_iota<<<(unsigned)((inner_units + 255) / 256 + 1), 256, 0, s>>>(inner_units, I(11), I(12));
  if (cudaGetLastError() != cudaSuccess) return MDRT_NB_CUDA_ERROR;
  return MDRT_NB_OK;
}

int32_t mdrtNbSetAbiStream(void *stream) {
  g_abi_stream = (cudaStream_t)stream;
  return MDRT_NB_OK;
}

void _mlir_ciface_mdrtCudaFFTForward3DF32(mdrtMemRef1D *real, mdrtMemRef1D *complex, int64_t k1, int64_t k2,
                                          int64_t k3) {
  if (!real || !complex) return note(MDRT_NB_INVALID_ARGUMENT, "a null descriptor");
  int32_t st = mdrtCudaFFTForward3DF32((const float *)real->aligned + real->offset,
                                       (float *)complex->aligned + complex->offset, k1, k2, k3, g_abi_stream);
  if (st != MDRT_NB_OK) note(st, "the forward transform failed");
}

void _mlir_ciface_mdrtCudaFFTBackward3DF32(mdrtMemRef1D *complex, mdrtMemRef1D *real, int64_t k1, int64_t k2,
                                           int64_t k3) {
  if (!real || !complex) return note(MDRT_NB_INVALID_ARGUMENT, "a null descriptor");
  int32_t st = mdrtCudaFFTBackward3DF32((float *)complex->aligned + complex->offset,
                                        (float *)real->aligned + real->offset, k1, k2, k3, g_abi_stream);
  if (st != MDRT_NB_OK) note(st, "the backward transform failed");
}

void _mlir_ciface_mdrtCudaFFTGaussianBackwardF32(mdrtMemRef1D *complex, mdrtMemRef1D *real, mdrtMemRef1D *tables,
                                                 int64_t k1, int64_t k2, int64_t k3) {
  if (!real || !complex || !tables) return note(MDRT_NB_INVALID_ARGUMENT, "a null descriptor");
  if (k1 < 1 || k2 < 1 || k3 < 1) return note(MDRT_NB_INVALID_ARGUMENT, "a grid of no points");
  float2 *spec = (float2 *)((float *)complex->aligned + complex->offset);
  int64_t total = k1 * k2 * (k3 / 2 + 1);
  unsigned blocks = (unsigned)std::min<int64_t>((total + 255) / 256, 148 * 8);
  abi_gaussian_scale<<<blocks, 256, 0, g_abi_stream>>>(k1, k2, k3, (const float *)tables->aligned + tables->offset,
                                                        spec);
  if (cudaGetLastError() != cudaSuccess) return note(MDRT_NB_CUDA_ERROR, "the Gaussian influence failed to launch");
  _mlir_ciface_mdrtCudaFFTBackward3DF32(complex, real, k1, k2, k3);
}

}  // extern "C"
