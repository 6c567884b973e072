// The C ABI of the batch of frames (include/mdrt_nb.h, mdrtNbBatch*): many
// independent systems of uneven sizes, each with its own cell and PME grid,
// evaluated by one launch of each kernel over all of them.
//
// MDIR evaluates the frames of an activation one after another (D251,
// docs/python-frames.md) and its device batch (D386, docs/driver.md:
// 1655-1700) loops over frames of one program; here the frames are laid
// end to end in one context (see mdrtNbBatch in nb_context.h), so the
// persistent pair kernel balances the units of all frames across the SMs
// and small frames do not leave the GPU idle.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/mdrt_nb.h"
#include "nb_context.h"

namespace {

int cuda_status(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return MDRT_NB_OK;
  fprintf(stderr, "mdrt_nb: %s: %s\n", what, cudaGetErrorString(e));
  return MDRT_NB_CUDA_ERROR;
}

#define CK(x)                                        \
  do {                                               \
    int s_ = cuda_status((x), #x);                   \
    if (s_) return s_;                               \
  } while (0)

template <typename T>
void bfree(T *&p) {
  if (p) cudaFree((void *)p);
  p = nullptr;
}

void drop_graph(mdrtNbBatch *b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  b->gkey = -1;
}

// The force evaluation's launches on `s` (no host wait, no allocation).
int batch_force_body(mdrtNbBatch *b, const double *x, uint32_t flags, double *forces, cudaStream_t s) {
  NbCtx &c = b->nb->c;
  bool energy = flags & MDRT_NB_ENERGY;
  bool pairs = !(flags & MDRT_NB_NO_PAIRS);
  bool excluded = !(flags & MDRT_NB_NO_EXCLUDED);
  bool pme = b->pme && !(flags & MDRT_NB_NO_PME) && c.beta > 0.0;
  if (!(flags & MDRT_NB_ACCUMULATE)) cudaMemsetAsync(forces, 0, sizeof(double) * 3 * c.n, s);
  nb_batch_gather_frames(*b, x, s);
  if (pairs) nb_batch_pairs_run(*b, energy, s);
  if (excluded) nb_batch_excluded_run(*b, energy, s);
  if (pme && nb_batch_pme_run(*b, energy, s)) return MDRT_NB_CUDA_ERROR;
  bool keep = c.pme.on;
  if (!pme) c.pme.on = false;
  nb_finish_forces(c, forces, 1, s);
  c.pme.on = keep;
  if (energy) nb_batch_energy_sums(*b, pairs, excluded, pme, s);
  return MDRT_NB_OK;
}

int check_boxes(const mdrtNbBatch &b, const double *boxes) {
  const NbCtx &c = b.nb->c;
  for (int f = 0; f < b.frames; ++f) {
    const double *L = boxes + 3 * f;
    for (int k = 0; k < 3; ++k)
      if (!(L[k] > 0.0) || !std::isfinite(L[k])) return MDRT_NB_INVALID_BOX;
    double least = std::min(L[0], std::min(L[1], L[2]));
    if (c.reach >= 0.999 * least || 2.0 * c.cutoff > least) return MDRT_NB_INVALID_BOX;
  }
  return MDRT_NB_OK;
}

}  // namespace

extern "C" {

int32_t mdrtNbBatchCreate(mdrtNbBatch **out, int32_t device, int32_t frames, const int64_t *atoms) {
  if (!out || frames < 1 || !atoms) return MDRT_NB_INVALID_ARGUMENT;
  *out = nullptr;
  int64_t total = 0;
  for (int f = 0; f < frames; ++f) {
    if (atoms[f] < 1) return MDRT_NB_INVALID_ARGUMENT;
    total += atoms[f];
  }
  if (total > (1ll << 26)) return MDRT_NB_INVALID_ARGUMENT;
  mdrtNbBatch *b = new mdrtNbBatch();
  int32_t s = mdrtNbCreate(&b->nb, device, total);
  if (s) {
    delete b;
    return s;
  }
  b->frames = frames;
  b->atom0.assign(frames + 1, 0);
  for (int f = 0; f < frames; ++f) b->atom0[f + 1] = b->atom0[f] + atoms[f];
  b->h_frames.assign(frames, NbFrameDev{});
  b->h_boxes.assign(3 * (size_t)frames, 0.0);
  std::vector<int32_t> af(total);
  for (int f = 0; f < frames; ++f)
    for (int64_t i = b->atom0[f]; i < b->atom0[f + 1]; ++i) af[i] = f;
  bool ok = cudaMalloc(&b->atom_frame, sizeof(int32_t) * total) == cudaSuccess &&
            cudaMalloc(&b->frame_energy, sizeof(double) * NB_E_SLOTS * frames) == cudaSuccess &&
            cudaMallocHost(&b->h_frame_energy, sizeof(double) * NB_E_SLOTS * frames) == cudaSuccess &&
            cudaMalloc(&b->d_excl_blk0, sizeof(int32_t) * (frames + 1)) == cudaSuccess;
  if (ok) {
    ok = cudaMemcpy(b->atom_frame, af.data(), sizeof(int32_t) * total, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemset(b->frame_energy, 0, sizeof(double) * NB_E_SLOTS * frames) == cudaSuccess &&
         cudaMemset(b->d_excl_blk0, 0, sizeof(int32_t) * (frames + 1)) == cudaSuccess;
  }
  b->h_excl_blk0.assign(frames + 1, 0);
  if (!ok) {
    mdrtNbBatchDestroy(b);
    return MDRT_NB_CUDA_ERROR;
  }
  *out = b;
  return MDRT_NB_OK;
}

int32_t mdrtNbBatchDestroy(mdrtNbBatch *b) {
  if (!b) return MDRT_NB_OK;
  if (b->nb) cudaSetDevice(b->nb->c.device);
  drop_graph(b);
  if (b->nb) nb_batch_pme_release(*b);
  bfree(b->frames_dev);
  bfree(b->atom_frame);
  bfree(b->atom_col);
  bfree(b->col_frame);
  bfree(b->group_frame);
  bfree(b->group_L);
  bfree(b->frame_units);
  bfree(b->search_scratch);
  bfree(b->excl_blk_frame);
  bfree(b->excl_blk_first);
  bfree(b->excl_frame_end);
  bfree(b->excl_part);
  bfree(b->d_excl_blk0);
  bfree(b->frame_energy);
  if (b->h_frame_energy) cudaFreeHost(b->h_frame_energy);
  if (b->nb) mdrtNbDestroy(b->nb);
  delete b;
  return MDRT_NB_OK;
}

int32_t mdrtNbBatchSetParticles(mdrtNbBatch *b, const double *charges, const int32_t *types, int32_t ntypes,
                                const double *sigma, const double *epsilon) {
  if (!b) return MDRT_NB_INVALID_ARGUMENT;
  drop_graph(b);
  return mdrtNbSetParticles(b->nb, charges, types, ntypes, sigma, epsilon);
}

int32_t mdrtNbBatchSetExclusions(mdrtNbBatch *b, const int32_t *offsets, const int32_t *partners) {
  if (!b || !offsets) return MDRT_NB_INVALID_ARGUMENT;
  NbCtx &c = b->nb->c;
  // every excluded pair inside one frame
  std::vector<int64_t> per_frame(b->frames, 0);
  for (int f = 0; f < b->frames; ++f)
    for (int64_t i = b->atom0[f]; i < b->atom0[f + 1]; ++i) {
      if (offsets[i + 1] < offsets[i]) return MDRT_NB_INVALID_ARGUMENT;
      for (int32_t k = offsets[i]; k < offsets[i + 1]; ++k) {
        int64_t j = partners[k];
        if (j < b->atom0[f] || j >= b->atom0[f + 1]) return MDRT_NB_INVALID_ARGUMENT;
        if (j > i) per_frame[f]++;
      }
    }
  drop_graph(b);
  int32_t s = mdrtNbSetExclusions(b->nb, offsets, partners);
  if (s) return s;
  // blocks of at most 256 pairs of one frame (the pairs are in order of i)
  std::vector<int32_t> blk_frame, blk_first, frame_end(b->frames), blk0(b->frames + 1, 0);
  int64_t first = 0;
  for (int f = 0; f < b->frames; ++f) {
    blk0[f] = (int32_t)blk_frame.size();
    for (int64_t k = 0; k < per_frame[f]; k += 256) {
      blk_frame.push_back(f);
      blk_first.push_back((int32_t)(first + k));
    }
    first += per_frame[f];
    frame_end[f] = (int32_t)first;
  }
  blk0[b->frames] = (int32_t)blk_frame.size();
  if (first != c.n_excl_pairs) return MDRT_NB_INVALID_ARGUMENT;
  b->excl_blocks = (int)blk_frame.size();
  b->h_excl_blk0 = blk0;
  bfree(b->excl_blk_frame);
  bfree(b->excl_blk_first);
  bfree(b->excl_frame_end);
  bfree(b->excl_part);
  size_t nb = std::max<size_t>(blk_frame.size(), 1);
  CK(cudaMalloc(&b->excl_blk_frame, sizeof(int32_t) * nb));
  CK(cudaMalloc(&b->excl_blk_first, sizeof(int32_t) * nb));
  CK(cudaMalloc(&b->excl_frame_end, sizeof(int32_t) * b->frames));
  CK(cudaMalloc(&b->excl_part, sizeof(double) * 8 * nb));
  if (!blk_frame.empty()) {
    CK(cudaMemcpy(b->excl_blk_frame, blk_frame.data(), sizeof(int32_t) * blk_frame.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b->excl_blk_first, blk_first.data(), sizeof(int32_t) * blk_first.size(), cudaMemcpyHostToDevice));
  }
  CK(cudaMemcpy(b->excl_frame_end, frame_end.data(), sizeof(int32_t) * b->frames, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(b->d_excl_blk0, blk0.data(), sizeof(int32_t) * (b->frames + 1), cudaMemcpyHostToDevice));
  return MDRT_NB_OK;
}

int32_t mdrtNbBatchSetInteraction(mdrtNbBatch *b, double cutoff, double reach, double beta, double coulomb) {
  if (!b) return MDRT_NB_INVALID_ARGUMENT;
  drop_graph(b);
  return mdrtNbSetInteraction(b->nb, cutoff, reach, beta, coulomb, 0, 0, 0.0);
}

int32_t mdrtNbBatchPmeSetup(mdrtNbBatch *b, const int32_t *grids, int32_t order) {
  if (!b || !grids) return MDRT_NB_INVALID_ARGUMENT;
  for (int f = 0; f < b->frames; ++f)
    for (int k = 0; k < 3; ++k)
      if (grids[3 * f + k] < 2 * order) return MDRT_NB_INVALID_ARGUMENT;
  CK(cudaSetDevice(b->nb->c.device));
  drop_graph(b);
  int s = nb_batch_pme_setup(*b, grids, order);
  if (s == -2) return MDRT_NB_UNSUPPORTED;
  if (s) return MDRT_NB_CUDA_ERROR;
  return MDRT_NB_OK;
}

int32_t mdrtNbBatchSetTuning(mdrtNbBatch *b, int32_t key, int32_t value) {
  if (!b) return MDRT_NB_INVALID_ARGUMENT;
  switch (key) {
    case MDRT_NB_TUNE_PAIR_BLOCKS_PER_SM:
      if (value < 1 || value > 4) return MDRT_NB_INVALID_ARGUMENT;
      b->nb->c.pair_blocks_per_sm = value;
      drop_graph(b);
      return MDRT_NB_OK;
    case MDRT_NB_TUNE_SEARCH_WARPS:
      if (value != 1 && value != 4) return MDRT_NB_INVALID_ARGUMENT;
      b->search_warps = value;
      return MDRT_NB_OK;
    case MDRT_NB_TUNE_STAGING_DEPTH:
      if (value != 1 && value != 2) return MDRT_NB_INVALID_ARGUMENT;
      b->nb->c.staging_depth = value;
      drop_graph(b);
      return MDRT_NB_OK;
  }
  return MDRT_NB_INVALID_ARGUMENT;
}

int32_t mdrtNbBatchBuild(mdrtNbBatch *b, const double *x, const double *boxes, void *stream, int32_t *sizes_out) {
  if (!b || !x || !boxes) return MDRT_NB_INVALID_ARGUMENT;
  int32_t s = check_boxes(*b, boxes);
  if (s) return s;
  NbCtx &c = b->nb->c;
  CK(cudaSetDevice(c.device));
  if (boxes != b->h_boxes.data()) std::memcpy(b->h_boxes.data(), boxes, sizeof(double) * 3 * b->frames);
  if (nb_batch_build_run(*b, x, (cudaStream_t)stream)) return MDRT_NB_CUDA_ERROR;
  // the lists ordered as a single system's build orders them
  if (nb_lj_partition_run(c, (cudaStream_t)stream)) return MDRT_NB_CUDA_ERROR;
  if (sizes_out)
    for (int k = 0; k < NB_SIZE_COUNT; ++k) sizes_out[k] = c.h_sizes[k];
  if (c.h_sizes[NB_SIZE_NAN] > 0) return MDRT_NB_NAN_POSITION;
  return MDRT_NB_OK;
}

int32_t mdrtNbBatchForce(mdrtNbBatch *b, const double *x, uint32_t flags, double *forces, void *stream) {
  if (!b || !x || !forces) return MDRT_NB_INVALID_ARGUMENT;
  NbCtx &c = b->nb->c;
  if (!c.built) return MDRT_NB_NOT_BUILT;
  cudaStream_t st = (cudaStream_t)stream;
  if (!(flags & MDRT_NB_GRAPH)) {
    int32_t s = batch_force_body(b, x, flags, forces, st);
    if (s) return s;
    CK(cudaGetLastError());
    return MDRT_NB_OK;
  }
  // the same launches as one CUDA graph, captured again when the buffers or
  // the arguments change (a build that grew, other pointers or flags)
  int64_t key = (int64_t)(uintptr_t)c.slab ^ ((int64_t)(uintptr_t)c.units << 1) ^ (c.places_cap << 3) ^
                (c.units_cap << 5) ^ (c.list_cap << 7) ^ ((int64_t)c.pair_blocks_per_sm << 11);
  uint32_t fl = flags & ~MDRT_NB_GRAPH;
  if (!b->exec || b->gx != x || b->gf != forces || b->gflags != fl || b->gkey != key) {
    drop_graph(b);
    cudaStream_t cap;
    CK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    int32_t s = MDRT_NB_OK;
    if (e == cudaSuccess) s = batch_force_body(b, x, fl, forces, cap);
    cudaGraph_t graph = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(cap, &graph);
    cudaStreamDestroy(cap);
    if (e != cudaSuccess || e2 != cudaSuccess || s) {
      if (graph) cudaGraphDestroy(graph);
      cudaGetLastError();
      return s ? s : MDRT_NB_CUDA_ERROR;
    }
    if (cudaGraphInstantiate(&b->exec, graph, 0) != cudaSuccess) {
      cudaGraphDestroy(graph);
      return MDRT_NB_CUDA_ERROR;
    }
    b->graph = graph;
    b->gx = x;
    b->gf = forces;
    b->gflags = fl;
    b->gkey = key;
  }
  CK(cudaGraphLaunch(b->exec, st));
  return MDRT_NB_OK;
}

int32_t mdrtNbBatchEnergies(mdrtNbBatch *b, void *stream, double *out) {
  if (!b || !out) return MDRT_NB_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  size_t bytes = sizeof(double) * NB_E_SLOTS * b->frames;
  CK(cudaMemcpyAsync(b->h_frame_energy, b->frame_energy, bytes, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  std::memcpy(out, b->h_frame_energy, bytes);
  return MDRT_NB_OK;
}

int32_t mdrtNbBatchConstants(mdrtNbBatch *b, double *out) {
  if (!b || !out) return MDRT_NB_INVALID_ARGUMENT;
  const NbCtx &c = b->nb->c;
  for (int f = 0; f < b->frames; ++f) {
    double sq = 0.0, net = 0.0;
    for (int64_t i = b->atom0[f]; i < b->atom0[f + 1]; ++i) {
      double q = i < (int64_t)c.h_q.size() ? c.h_q[i] : 0.0;
      sq += q * q;
      net += q;
    }
    const double *L = &b->h_boxes[3 * f];
    double V = L[0] * L[1] * L[2];
    out[2 * f] = c.beta > 0 ? -c.coulomb * c.beta / std::sqrt(M_PI) * sq : 0.0;
    out[2 * f + 1] = (c.beta > 0 && V > 0) ? -c.coulomb * M_PI * net * net / (2.0 * V * c.beta * c.beta) : 0.0;
  }
  return MDRT_NB_OK;
}

int32_t mdrtNbBatchAutotune(mdrtNbBatch *b, const double *x, double *forces, void *stream, int32_t *choice) {
  if (!b || !x || !forces) return MDRT_NB_INVALID_ARGUMENT;
  NbCtx &c = b->nb->c;
  cudaStream_t st = (cudaStream_t)stream;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  float best = 1e30f;
  int best_w = b->search_warps, best_p = c.pair_blocks_per_sm, best_d = c.staging_depth;
  int32_t status = MDRT_NB_OK;
  for (int w : {4, 1}) {
    for (int trial = 0; trial < 8; ++trial) {
      int pb = 4 - trial / 2, depth = 1 + trial % 2;
      b->search_warps = w;
      c.pair_blocks_per_sm = pb;
      c.staging_depth = depth;
      drop_graph(b);
      // a warm-up, then three timed builds + evaluations
      status = mdrtNbBatchBuild(b, x, b->h_boxes.data(), stream, nullptr);
      if (!status) status = batch_force_body(b, x, MDRT_NB_ENERGY, forces, st);
      if (status) break;
      cudaEventRecord(e0, st);
      for (int r = 0; r < 3 && !status; ++r) {
        if (nb_batch_build_run(*b, x, st)) status = MDRT_NB_CUDA_ERROR;
        if (!status) status = batch_force_body(b, x, MDRT_NB_ENERGY, forces, st);
      }
      cudaEventRecord(e1, st);
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (!status && ms < best) {
        best = ms;
        best_w = w;
        best_p = pb;
        best_d = depth;
      }
    }
    if (status) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->search_warps = best_w;
  c.pair_blocks_per_sm = best_p;
  c.staging_depth = best_d;
  if (best_w == 1) {  // a warp a group stages nothing
    bfree(b->search_scratch);
    b->search_scratch_entries = 0;
  }
  drop_graph(b);
  if (choice) {
    choice[0] = best_w;
    choice[1] = best_p;
    choice[2] = best_d;
  }
  return status;
}

}  // extern "C"
