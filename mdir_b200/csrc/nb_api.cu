// The C ABI of include/mdrt_nb.h over the host context NbCtx.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
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
void nb_free(T *&p) {
  if (p) cudaFree((void *)p);
  p = nullptr;
}

int check_box(const NbCtx &c, const double box[3]) {
  if (!box) return MDRT_NB_INVALID_ARGUMENT;
  for (int k = 0; k < 3; ++k)
    if (!(box[k] > 0.0) || !std::isfinite(box[k])) return MDRT_NB_INVALID_BOX;
  double least = std::min(box[0], std::min(box[1], box[2]));
  // MDIR refuses a pairlist distance above 0.999 of the least edge
  // (docs/neighbor-groups.md, Section 5.2) and a cutoff above half of it.
  if (c.reach >= 0.999 * least || 2.0 * c.cutoff > least) return MDRT_NB_INVALID_BOX;
  return MDRT_NB_OK;
}

// The squared largest displacement of frame blockIdx.y from the positions of
// the last build, under the minimum image, as the bits of a non-negative
// double (which order like the integers); a coordinate that is not finite
// counts as infinitely far.
__global__ void nb_frame_drift(int64_t n, const double *__restrict__ frames, const double *__restrict__ ref,
                               double Lx, double Ly, double Lz, unsigned long long *__restrict__ out) {
  const double *x = frames + (int64_t)blockIdx.y * 3 * n;
  double m = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double d0 = x[3 * i] - ref[3 * i], d1 = x[3 * i + 1] - ref[3 * i + 1], d2 = x[3 * i + 2] - ref[3 * i + 2];
    d0 -= Lx * rint(d0 / Lx);
    d1 -= Ly * rint(d1 / Ly);
    d2 -= Lz * rint(d2 / Lz);
    double r2 = d0 * d0 + d1 * d1 + d2 * d2;
    m = r2 == r2 ? fmax(m, r2) : INFINITY;
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out + blockIdx.y, (unsigned long long)__double_as_longlong(m));
}

// ---- the graphs of the frames entries ----
// A frames call launches about a dozen kernels a frame, and for a frame of a
// few ten thousand atoms the host's launch rate, not the GPU, bounds it.
// The launches of a call are therefore kept as a CUDA graph under a key of
// the call's arguments and the bytes of the context as the call found it:
// every buffer pointer, capacity, tuning value, interaction parameter and
// build count of NbCtx, so that any change of the context that alters what
// the launches are (a build, a growth, new tuning, a new cell) changes the
// key.  The graph reads the frames, the particle tables and the lists at its
// launch.  The host arrays of NbCtx (h_q and the like) are not in the key:
// the launches kept here take no argument computed from them.
#define NB_FRAME_GRAPHS 8

std::vector<unsigned char> nb_frames_key(const NbCtx &c, const uint64_t *args, int nargs) {
  std::vector<unsigned char> key(sizeof(uint64_t) * nargs + sizeof(NbCtx));
  std::memcpy(key.data(), args, sizeof(uint64_t) * nargs);
  const unsigned char *b = reinterpret_cast<const unsigned char *>(&c);
  std::copy(b, b + sizeof(NbCtx), key.begin() + sizeof(uint64_t) * nargs);
  return key;
}

uint64_t nb_bits(double v) {
  uint64_t u;
  std::memcpy(&u, &v, sizeof(u));
  return u;
}

uint64_t nb_bits(const void *p) { return (uint64_t)(uintptr_t)p; }

// Runs `run(stream)` (the launches of one frames call) for the caller's
// stream st: a key met before with a graph is one graph launch; a key met
// once before is captured now, on the context's own stream, and launched;
// a new key runs directly (its lazy allocations and tables then happen
// outside any capture) and is remembered.  The least recently used of more
// than NB_FRAME_GRAPHS keys is dropped (a graph still running is freed when
// it completes).
template <class Run>
int32_t nb_frames_graph(mdrtNb *ctx, const uint64_t *args, int nargs, cudaStream_t st, Run &&run) {
  NbCtx &c = ctx->c;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (!c.frame_graphs) return run(st);
  CK(cudaStreamIsCapturing(st, &cs));
  if (cs != cudaStreamCaptureStatusNone) return run(st);
  std::vector<unsigned char> key = nb_frames_key(c, args, nargs);
  NbFrameGraph *hit = nullptr;
  for (auto &g : ctx->graphs)
    if (g.key == key) hit = &g;
  if (!hit) {
    int32_t s = run(st);
    if (s) return s;
    if ((int)ctx->graphs.size() >= NB_FRAME_GRAPHS) {
      auto old = std::min_element(ctx->graphs.begin(), ctx->graphs.end(),
                                  [](const NbFrameGraph &a, const NbFrameGraph &b) { return a.used < b.used; });
      if (old->exec) cudaGraphExecDestroy(old->exec);
      ctx->graphs.erase(old);
    }
    NbFrameGraph g;
    g.key = std::move(key);
    g.used = ++ctx->graph_clock;
    ctx->graphs.push_back(std::move(g));
    return MDRT_NB_OK;
  }
  hit->used = ++ctx->graph_clock;
  if (!hit->exec) {
    if (!ctx->capture) CK(cudaStreamCreateWithFlags(&ctx->capture, cudaStreamNonBlocking));
    CK(cudaStreamBeginCapture(ctx->capture, cudaStreamCaptureModeThreadLocal));
    int32_t s = run(ctx->capture);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(ctx->capture, &graph);
    if (s || e != cudaSuccess || !graph) {
      if (graph) cudaGraphDestroy(graph);
      cudaGetLastError();
      return s ? s : cuda_status(e, "cudaStreamEndCapture");
    }
    e = cudaGraphInstantiate(&hit->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      hit->exec = nullptr;
      return cuda_status(e, "cudaGraphInstantiate");
    }
    ctx->graph_captures++;
    CK(cudaGraphLaunch(hit->exec, st));
    // the capture ran as the call before it, so it left the context as it
    // was; if not, the graph holds work of that change and is not kept
    if (nb_frames_key(c, args, nargs) != hit->key) {
      cudaGraphExecDestroy(hit->exec);
      hit->exec = nullptr;
    }
    return MDRT_NB_OK;
  }
  CK(cudaGraphLaunch(hit->exec, st));
  ctx->graph_replays++;
  return MDRT_NB_OK;
}

}  // namespace

extern "C" {

int32_t mdrtNbVersion(void) { return MDRT_NB_ABI_VERSION; }

const char *mdrtNbStatusString(int32_t s) {
  switch (s) {
    case MDRT_NB_OK: return "ok";
    case MDRT_NB_GROW: return "a buffer was too small and has grown; call again";
    case MDRT_NB_NAN_POSITION: return "positions that are not finite or are far outside the cell";
    case MDRT_NB_INVALID_BOX: return "the reach is at least 0.999 of the least edge, the cutoff above half of it, or an edge is not positive";
    case MDRT_NB_CUDA_ERROR: return "a CUDA call failed";
    case MDRT_NB_TIMEOUT: return "a device wait ran out of time";
    case MDRT_NB_INVALID_ARGUMENT: return "invalid argument";
    case MDRT_NB_UNSUPPORTED: return "unsupported";
    case MDRT_NB_OVERFLOW: return "a fixed-point accumulator went out of range";
    case MDRT_NB_NOT_BUILT: return "no neighbor build yet";
  }
  return "unknown status";
}

int32_t mdrtNbCreate(mdrtNb **out, int32_t device, int64_t particles) {
  if (!out || particles <= 0 || particles > (1ll << 26)) return MDRT_NB_INVALID_ARGUMENT;
  *out = nullptr;
  CK(cudaSetDevice(device));
  mdrtNb *ctx = new mdrtNb();
  NbCtx &c = ctx->c;
  c.device = device;
  c.n = particles;
  if (cudaMalloc(&c.sizes, sizeof(int32_t) * NB_SIZE_COUNT) != cudaSuccess ||
      cudaMallocHost(&c.h_sizes, sizeof(int32_t) * NB_SIZE_COUNT) != cudaSuccess ||
      cudaMalloc(&c.status, sizeof(int32_t)) != cudaSuccess ||
      cudaMalloc(&c.energy, sizeof(double) * NB_E_SLOTS) != cudaSuccess ||
      cudaMallocHost(&c.h_energy, sizeof(double) * NB_E_SLOTS) != cudaSuccess) {
    mdrtNbDestroy(ctx);
    return MDRT_NB_CUDA_ERROR;
  }
  cudaMemset(c.sizes, 0, sizeof(int32_t) * NB_SIZE_COUNT);
  cudaMemset(c.status, 0, sizeof(int32_t));
  cudaMemset(c.energy, 0, sizeof(double) * NB_E_SLOTS);
  // default particle table: no charge, one type of no interaction
  std::vector<double> q(particles, 0.0);
  std::vector<int32_t> t(particles, 0);
  double sg = 0.3, ep = 0.0;
  int32_t s = mdrtNbSetParticles(ctx, q.data(), t.data(), 1, &sg, &ep);
  if (s) {
    mdrtNbDestroy(ctx);
    return s;
  }
  *out = ctx;
  return MDRT_NB_OK;
}

int32_t mdrtNbDestroy(mdrtNb *ctx) {
  if (!ctx) return MDRT_NB_OK;
  NbCtx &c = ctx->c;
  cudaSetDevice(c.device);
  for (auto &g : ctx->graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  ctx->graphs.clear();
  if (ctx->capture) cudaStreamDestroy(ctx->capture);
  nb_pme_release(c);
  nb_free(c.q); nb_free(c.type); nb_free(c.lj); nb_free(c.ljf); nb_free(c.sigeps);
  nb_free(c.lj_on); nb_free(c.counts_lj);
  nb_free(c.adj_g); nb_free(c.adj_q); nb_free(c.adj_types); nb_free(c.x_build); nb_free(c.drift);
  if (c.h_drift) cudaFreeHost(c.h_drift);
  if (ctx->drift_done) cudaEventDestroy(ctx->drift_done);
  nb_free(c.excl_off); nb_free(c.excl); nb_free(c.excl_pairs); nb_free(c.excl_partials);
  nb_free(c.order); nb_free(c.place_of); nb_free(c.shift); nb_free(c.xw);
  nb_free(c.box_lo); nb_free(c.box_hi); nb_free(c.group_start); nb_free(c.group_col);
  nb_free(c.slab); nb_free(c.counts); nb_free(c.unit_n); nb_free(c.unit_start); nb_free(c.units);
  nb_free(c.sizes); nb_free(c.status);
  nb_free(c.key); nb_free(c.bin_count); nb_free(c.bin_start); nb_free(c.bin_fill);
  nb_free(c.sorted); nb_free(c.col_groups); nb_free(c.scan_scratch);
  nb_free(c.atom_xw); nb_free(c.atom_shift);
  nb_free(c.xq); nb_free(c.xq_lo); nb_free(c.typ_p); nb_free(c.acc); nb_free(c.acc_fixed);
  nb_free(c.unit_partials); nb_free(c.energy);
  nb_free(c.slab_in); nb_free(c.counts_in); nb_free(c.unit_n_in); nb_free(c.unit_start_in);
  nb_free(c.units_in); nb_free(c.sizes_in); nb_free(c.one);
  if (c.h_sizes) cudaFreeHost(c.h_sizes);
  if (c.h_energy) cudaFreeHost(c.h_energy);
  delete ctx;
  return MDRT_NB_OK;
}

int32_t mdrtNbSetParticles(mdrtNb *ctx, const double *charges, const int32_t *types, int32_t ntypes,
                           const double *sigma, const double *epsilon) {
  if (!ctx || !charges || !types || ntypes < 1 || ntypes > 32 || !sigma || !epsilon)
    return MDRT_NB_INVALID_ARGUMENT;
  NbCtx &c = ctx->c;
  CK(cudaSetDevice(c.device));
  for (int64_t i = 0; i < c.n; ++i)
    if (types[i] < 0 || types[i] >= ntypes || !std::isfinite(charges[i])) return MDRT_NB_INVALID_ARGUMENT;
  c.h_q.assign(charges, charges + c.n);
  c.h_type.assign(types, types + c.n);
  c.h_lj.resize((size_t)ntypes * ntypes);
  c.h_c6.resize((size_t)ntypes * ntypes);
  std::vector<float2> se((size_t)ntypes * ntypes);
  for (int a = 0; a < ntypes * ntypes; ++a) {
    se[a] = make_float2((float)sigma[a], (float)epsilon[a]);
    double s6 = std::pow(sigma[a], 6.0);
    c.h_c6[a] = 4.0 * epsilon[a] * s6;
    c.h_lj[a] = make_float2((float)(4.0 * epsilon[a] * s6), (float)(4.0 * epsilon[a] * s6 * s6));
  }
  // Does the table factorize, c_ab = sqrt(c_aa c_bb) for both c6 and c12
  // (one LJ type, or geometric mixing)?  Then the pair kernel multiplies
  // per-type factors instead of looking the pair up.
  std::vector<float2> factors(ntypes);
  bool geom = true;
  for (int a = 0; a < ntypes; ++a) {
    double c6 = c.h_c6[a * ntypes + a], c12 = 4.0 * epsilon[a * ntypes + a] * std::pow(sigma[a * ntypes + a], 12.0);
    if (c6 < 0 || c12 < 0) geom = false;
    factors[a] = make_float2((float)std::sqrt(std::max(c6, 0.0)), (float)std::sqrt(std::max(c12, 0.0)));
  }
  for (int a = 0; a < ntypes && geom; ++a)
    for (int b = 0; b < ntypes && geom; ++b) {
      double c6 = c.h_c6[a * ntypes + b];
      double c12 = 4.0 * epsilon[a * ntypes + b] * std::pow(sigma[a * ntypes + b], 12.0);
      double g6 = (double)factors[a].x * factors[b].x, g12 = (double)factors[a].y * factors[b].y;
      if (std::fabs(c6 - g6) > 1e-6 * std::fabs(c6) + 1e-30 || std::fabs(c12 - g12) > 1e-6 * std::fabs(c12) + 1e-30)
        geom = false;
    }
  c.lj_geom = geom;
  std::vector<float> qf(charges, charges + c.n);
  // the tables keep their buffers (sized for 32 types) from one call to the
  // next, so that new parameters leave the kernels' arguments as they were
  // (and the frames entries' graphs valid); the work in flight on any
  // stream finishes before they are written
  CK(cudaDeviceSynchronize());
  if (!c.q) CK(cudaMalloc(&c.q, sizeof(float) * c.n));
  if (!c.type) CK(cudaMalloc(&c.type, sizeof(int32_t) * c.n));
  if (!c.ljf) CK(cudaMalloc(&c.ljf, sizeof(float2) * 32));
  if (!c.lj) CK(cudaMalloc(&c.lj, sizeof(float2) * 32 * 32));
  if (!c.sigeps) CK(cudaMalloc(&c.sigeps, sizeof(float2) * 32 * 32));
  if (!c.lj_on) CK(cudaMalloc(&c.lj_on, sizeof(int32_t) * 32));
  int32_t on[32] = {0};
  uint32_t mask = 0;
  for (int a = 0; a < ntypes; ++a)
    for (int b = 0; b < ntypes; ++b)
      if (epsilon[a * ntypes + b] != 0.0) on[a] = 1;
  for (int a = 0; a < ntypes; ++a) mask |= on[a] ? (1u << a) : 0u;
  CK(cudaMemcpy(c.lj_on, on, sizeof(on), cudaMemcpyHostToDevice));
  c.lj_mask = mask;
  CK(cudaMemcpy(c.ljf, factors.data(), sizeof(float2) * ntypes, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c.sigeps, se.data(), sizeof(float2) * ntypes * ntypes, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c.q, qf.data(), sizeof(float) * c.n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c.type, types, sizeof(int32_t) * c.n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c.lj, c.h_lj.data(), sizeof(float2) * ntypes * ntypes, cudaMemcpyHostToDevice));
  c.ntypes = ntypes;
  return MDRT_NB_OK;
}

int32_t mdrtNbSetExclusions(mdrtNb *ctx, const int32_t *offsets, const int32_t *partners) {
  if (!ctx || !offsets) return MDRT_NB_INVALID_ARGUMENT;
  NbCtx &c = ctx->c;
  CK(cudaSetDevice(c.device));
  int64_t total = offsets[c.n];
  if (offsets[0] != 0 || total < 0 || (total > 0 && !partners)) return MDRT_NB_INVALID_ARGUMENT;
  std::vector<int32_t> pairs;
  for (int64_t i = 0; i < c.n; ++i) {
    if (offsets[i + 1] < offsets[i]) return MDRT_NB_INVALID_ARGUMENT;
    for (int32_t k = offsets[i]; k < offsets[i + 1]; ++k) {
      int32_t j = partners[k];
      if (j < 0 || j >= c.n || j == i) return MDRT_NB_INVALID_ARGUMENT;
      if (j > i) {
        pairs.push_back((int32_t)i);
        pairs.push_back(j);
      }
    }
  }
  nb_free(c.excl_off);
  nb_free(c.excl);
  nb_free(c.excl_pairs);
  nb_free(c.excl_partials);
  CK(cudaMalloc(&c.excl_off, sizeof(int32_t) * (c.n + 1)));
  CK(cudaMemcpy(c.excl_off, offsets, sizeof(int32_t) * (c.n + 1), cudaMemcpyHostToDevice));
  CK(cudaMalloc(&c.excl, sizeof(int32_t) * std::max<int64_t>(total, 1)));
  if (total > 0) CK(cudaMemcpy(c.excl, partners, sizeof(int32_t) * total, cudaMemcpyHostToDevice));
  c.n_excl_pairs = (int64_t)pairs.size() / 2;
  CK(cudaMalloc(&c.excl_pairs, sizeof(int32_t) * std::max<size_t>(pairs.size(), 2)));
  if (!pairs.empty())
    CK(cudaMemcpy(c.excl_pairs, pairs.data(), sizeof(int32_t) * pairs.size(), cudaMemcpyHostToDevice));
  int64_t blocks = std::max<int64_t>(1, (c.n_excl_pairs + 255) / 256);
  CK(cudaMalloc(&c.excl_partials, sizeof(double) * 8 * blocks));
  c.built = false;  // the lists depend on the exclusions
  return MDRT_NB_OK;
}

int32_t mdrtNbSetInteraction(mdrtNb *ctx, double cutoff, double reach, double beta, double coulomb,
                             int32_t coulomb_shift, int32_t lj_switch, double switch_distance) {
  if (!ctx || !(cutoff > 0) || !(reach >= cutoff) || !(beta >= 0) || !std::isfinite(coulomb))
    return MDRT_NB_INVALID_ARGUMENT;
  if (lj_switch < 0 || lj_switch > 2) return MDRT_NB_INVALID_ARGUMENT;
  if (lj_switch && !(switch_distance >= 0 && switch_distance < cutoff)) return MDRT_NB_INVALID_ARGUMENT;
  NbCtx &c = ctx->c;
  c.cutoff = cutoff;
  if (reach != c.reach) c.built = false;
  c.reach = reach;
  c.beta = beta;
  c.coulomb = coulomb;
  c.coulomb_shift = coulomb_shift;
  c.lj_switch = lj_switch;
  c.switch_distance = switch_distance;
  return MDRT_NB_OK;
}

int32_t mdrtNbSetTuning(mdrtNb *ctx, int32_t key, int32_t value) {
  if (!ctx) return MDRT_NB_INVALID_ARGUMENT;
  switch (key) {
    case MDRT_NB_TUNE_PAIR_BLOCKS_PER_SM:
      if (value < 1 || value > 4) return MDRT_NB_INVALID_ARGUMENT;
      ctx->c.pair_blocks_per_sm = value;
      return MDRT_NB_OK;
    case MDRT_NB_TUNE_STAGING_DEPTH:
      if (value != 1 && value != 2) return MDRT_NB_INVALID_ARGUMENT;
      ctx->c.staging_depth = value;
      return MDRT_NB_OK;
    case MDRT_NB_TUNE_FUSED_PRUNE:
      if (value < 0 || value > 2) return MDRT_NB_INVALID_ARGUMENT;
      ctx->c.fused_prune = value;
      return MDRT_NB_OK;
    case MDRT_NB_TUNE_PAIR_SMS:
      if (value < 0 || value > 4096) return MDRT_NB_INVALID_ARGUMENT;
      ctx->c.pair_sms = value;
      return MDRT_NB_OK;
    case MDRT_NB_TUNE_PME_FFT:
      if (value != 0 && value != 1) return MDRT_NB_INVALID_ARGUMENT;
      ctx->c.pme_fft = value;
      return MDRT_NB_OK;
    case MDRT_NB_TUNE_PME_SPREAD:
      if (value < 0 || value > 2) return MDRT_NB_INVALID_ARGUMENT;
      ctx->c.pme_spread = value;
      return MDRT_NB_OK;
    case MDRT_NB_TUNE_FRAME_GRAPHS:
      if (value != 0 && value != 1) return MDRT_NB_INVALID_ARGUMENT;
      ctx->c.frame_graphs = value;
      return MDRT_NB_OK;
  }
  return MDRT_NB_INVALID_ARGUMENT;
}

int32_t mdrtNbSetPrunedReach(mdrtNb *ctx, double pruned_distance) {
  if (!ctx || !(pruned_distance == 0.0 || (pruned_distance >= ctx->c.cutoff && pruned_distance <= ctx->c.reach)))
    return MDRT_NB_INVALID_ARGUMENT;
  NbCtx &c = ctx->c;
  if (pruned_distance >= c.reach) pruned_distance = 0.0;  // no tighter than the outer list: one list
  c.inner_reach = pruned_distance;
  c.inner_valid = false;
  if (c.inner_reach > 0.0 && c.built) {
    int64_t key = c.groups_cap * 1000003 + c.list_cap * 7 + c.units_cap;
    if (key != c.inner_key || !c.slab_in) {
      if (nb_reserve_inner(c)) return MDRT_NB_CUDA_ERROR;
      c.inner_key = key;
    }
  }
  return MDRT_NB_OK;
}

int32_t mdrtNbPrune(mdrtNb *ctx, const double *x, const double box[3], void *stream) {
  if (!ctx || !x || !box) return MDRT_NB_INVALID_ARGUMENT;
  NbCtx &c = ctx->c;
  if (!c.built) return MDRT_NB_NOT_BUILT;
  if (c.inner_reach <= 0.0) return MDRT_NB_OK;
  cudaStream_t st = (cudaStream_t)stream;
  nb_gather_frames(c, x, box, st);
  nb_prune_run(c, box, st);
  c.inner_valid = true;
  c.prunes++;
  CK(cudaGetLastError());
  return MDRT_NB_OK;
}

int32_t mdrtNbSetDeterministic(mdrtNb *ctx, int32_t on) {
  if (!ctx) return MDRT_NB_INVALID_ARGUMENT;
  ctx->c.deterministic = on != 0;
  return MDRT_NB_OK;
}

int32_t mdrtPmeSetup(mdrtNb *ctx, int32_t k1, int32_t k2, int32_t k3, int32_t order) {
  if (!ctx) return MDRT_NB_INVALID_ARGUMENT;
  NbCtx &c = ctx->c;
  CK(cudaSetDevice(c.device));
  if (k1 == 0 && k2 == 0 && k3 == 0) {
    nb_pme_release(c);
    return MDRT_NB_OK;
  }
  if (k1 < 2 * order || k2 < 2 * order || k3 < 2 * order) return MDRT_NB_INVALID_ARGUMENT;
  int s = nb_pme_setup(c, k1, k2, k3, order);
  if (s == -2) return MDRT_NB_UNSUPPORTED;
  if (s != 0) return MDRT_NB_CUDA_ERROR;
  return MDRT_NB_OK;
}

// The build in the cell of c.tilt (set by the caller): see mdrtNbBuild.
static int32_t nb_build_entry(mdrtNb *ctx, const double *x, int64_t n, const double box[3], double reach,
                              void *stream, int32_t *sizes_out);

int32_t mdrtNbBuild(mdrtNb *ctx, const double *x, int64_t n, const double box[3], double reach,
                    void *stream, int32_t *sizes_out) {
  if (!ctx || !x) return MDRT_NB_INVALID_ARGUMENT;
  for (double &t : ctx->c.tilt) t = 0.0;
  return nb_build_entry(ctx, x, n, box, reach, stream, sizes_out);
}

// A triclinic cell (ax, by, cz, bx, cx, cy) in MDIR's reduced form:
// |bx| <= ax/2, |cx| <= ax/2, |cy| <= by/2.
static int check_cell(const double cell[6]) {
  if (!cell) return MDRT_NB_INVALID_ARGUMENT;
  for (int k = 0; k < 6; ++k)
    if (!std::isfinite(cell[k])) return MDRT_NB_INVALID_BOX;
  const double slack = 1.0 + 1e-9;
  if (std::fabs(cell[3]) > 0.5 * cell[0] * slack || std::fabs(cell[4]) > 0.5 * cell[0] * slack ||
      std::fabs(cell[5]) > 0.5 * cell[1] * slack)
    return MDRT_NB_INVALID_BOX;
  return MDRT_NB_OK;
}

int32_t mdrtNbBuildTriclinic(mdrtNb *ctx, const double *x, int64_t n, const double cell[6], double reach,
                             void *stream, int32_t *sizes_out) {
  if (!ctx || !x) return MDRT_NB_INVALID_ARGUMENT;
  int s = check_cell(cell);
  if (s) return s;
  for (int k = 0; k < 3; ++k) ctx->c.tilt[k] = cell[3 + k];
  return nb_build_entry(ctx, x, n, cell, reach, stream, sizes_out);
}

static int32_t nb_build_entry(mdrtNb *ctx, const double *x, int64_t n, const double box[3], double reach,
                              void *stream, int32_t *sizes_out) {
  NbCtx &c = ctx->c;
  if (n != c.n) return MDRT_NB_INVALID_ARGUMENT;
  if (reach > 0 && reach != c.reach) {
    if (reach < c.cutoff) return MDRT_NB_INVALID_ARGUMENT;
    c.reach = reach;
  }
  int s = check_box(c, box);
  if (s) return s;
  CK(cudaSetDevice(c.device));
  cudaStream_t st = (cudaStream_t)stream;
  if (nb_build_run(c, x, box, st)) return MDRT_NB_CUDA_ERROR;
  if (nb_lj_partition_run(c, st)) return MDRT_NB_CUDA_ERROR;
  for (int k = 0; k < 3; ++k) c.tilt_built[k] = c.tilt[k];
  if (!c.x_build) CK(cudaMalloc(&c.x_build, sizeof(double) * 3 * c.n));
  CK(cudaMemcpyAsync(c.x_build, x, sizeof(double) * 3 * c.n, cudaMemcpyDeviceToDevice, st));
  if (sizes_out)
    for (int k = 0; k < NB_SIZE_COUNT; ++k) sizes_out[k] = c.h_sizes[k];
  if (c.h_sizes[NB_SIZE_NAN] > 0) return MDRT_NB_NAN_POSITION;
  return MDRT_NB_OK;
}

static int32_t nb_force_entry(mdrtNb *ctx, const double *x, const double box[3], uint32_t flags, double *forces,
                              void *stream);

int32_t mdrtNbForce(mdrtNb *ctx, const double *x, const double box[3], uint32_t flags, double *forces,
                    void *stream) {
  if (!ctx || !x || !forces) return MDRT_NB_INVALID_ARGUMENT;
  if (nb_triclinic(ctx->c)) return MDRT_NB_INVALID_BOX;  // built in a triclinic cell
  return nb_force_entry(ctx, x, box, flags, forces, stream);
}

int32_t mdrtNbForceTriclinic(mdrtNb *ctx, const double *x, const double cell[6], uint32_t flags, double *forces,
                             void *stream) {
  if (!ctx || !x || !forces) return MDRT_NB_INVALID_ARGUMENT;
  int s = check_cell(cell);
  if (s) return s;
  for (int k = 0; k < 3; ++k)
    if (cell[3 + k] != ctx->c.tilt_built[k]) return MDRT_NB_INVALID_BOX;  // a cell change needs a build
  return nb_force_entry(ctx, x, cell, flags, forces, stream);
}

static int32_t nb_force_entry(mdrtNb *ctx, const double *x, const double box[3], uint32_t flags, double *forces,
                              void *stream) {
  NbCtx &c = ctx->c;
  if (!c.built) return MDRT_NB_NOT_BUILT;
  int s = check_box(c, box);
  if (s) return s;
  for (int k = 0; k < 3; ++k)
    if (box[k] != c.box_built[k]) return MDRT_NB_INVALID_BOX;  // a cell change needs a build
  cudaStream_t st = (cudaStream_t)stream;
  bool energy = flags & MDRT_NB_ENERGY;
  bool pairs = !(flags & MDRT_NB_NO_PAIRS);
  bool excluded = !(flags & MDRT_NB_NO_EXCLUDED);
  bool pme = c.pme.on && !(flags & MDRT_NB_NO_PME) && c.beta > 0.0;
  if (!(flags & MDRT_NB_ACCUMULATE)) CK(cudaMemsetAsync(forces, 0, sizeof(double) * 3 * c.n, st));
  if (energy) CK(cudaMemsetAsync(c.energy, 0, sizeof(double) * NB_E_SLOTS, st));
  nb_gather_frames(c, x, box, st);
  bool pairs_done = false;
  if ((flags & MDRT_NB_PRUNE) && c.inner_reach > 0.0) {
    // the pruning at x, and, for forces outside the deterministic mode, the
    // pairs of the pruned lists in the same kernel (MDIR D284)
    if (pairs && !energy && !c.deterministic && sizeof(int2) * (size_t)c.list_cap <= NB_FUSED_STAGE_MAX) {
      if (!c.one) {
        CK(cudaMalloc(&c.one, sizeof(int32_t)));
        int32_t h_one = 1;
        CK(cudaMemcpy(c.one, &h_one, sizeof(int32_t), cudaMemcpyHostToDevice));
      }
      CK(cudaMemsetAsync(c.sizes_in + NB_SIZE_UNITS, 0, sizeof(int32_t), st));  // the blocks claim their units
      nb_prune_pairs_run(c, box, c.one, x, nullptr, nullptr, c.sizes_in + NB_SIZE_UNITS, st, nullptr);
      pairs_done = true;
    } else {
      nb_prune_run(c, box, st);
    }
    c.inner_valid = true;
    c.prunes++;
  }
  if (pairs && !pairs_done) nb_pairs_run(c, box, energy, st);
  if (excluded) nb_excluded_run(c, box, energy, st);
  if (energy && (pairs || excluded)) nb_reduce_energy(c, pairs, excluded, st);
  if (pme) {
    if (nb_pme_run(c, box, energy, (flags & MDRT_NB_POTENTIAL) != 0, st)) return MDRT_NB_CUDA_ERROR;
  }
  bool keep_pme = c.pme.on;
  if (!pme) c.pme.on = false;  // finish without the PME forces of a skipped sum
  nb_finish_forces(c, forces, 1, st);
  c.pme.on = keep_pme;
  CK(cudaGetLastError());
  return MDRT_NB_OK;
}

// The checks of the gradient entries and the adjoint's scratch (allocated
// here, outside any capture).
static int32_t nb_gradient_ready(mdrtNb *ctx, const double *x, const double box[3], const double *cotangent,
                                 int32_t mode, const float *phi, double *dq, double *dtable) {
  if (!ctx || !x || !box || !dq || !dtable) return MDRT_NB_INVALID_ARGUMENT;
  if (mode != MDRT_NB_GRAD_PRODUCT && mode != MDRT_NB_GRAD_ENERGY) return MDRT_NB_INVALID_ARGUMENT;
  if (mode == MDRT_NB_GRAD_PRODUCT && !cotangent) return MDRT_NB_INVALID_ARGUMENT;
  NbCtx &c = ctx->c;
  if (!c.built) return MDRT_NB_NOT_BUILT;
  if (nb_triclinic(c)) return MDRT_NB_UNSUPPORTED;  // the adjoint runs in orthorhombic cells
  int s = check_box(c, box);
  if (s) return s;
  for (int k = 0; k < 3; ++k)
    if (box[k] != c.box_built[k]) return MDRT_NB_INVALID_BOX;
  // the switched Lennard-Jones form has no adjoint here
  if (c.lj_switch) return MDRT_NB_UNSUPPORTED;
  if (phi && !c.pme.on) return MDRT_NB_INVALID_ARGUMENT;
  CK(cudaSetDevice(c.device));
  if (nb_adjoint_reserve(c)) return MDRT_NB_CUDA_ERROR;
  return MDRT_NB_OK;
}

int32_t mdrtNbForceFrames(mdrtNb *ctx, const double *x, int64_t x_stride, int64_t count, const double box[3],
                          uint32_t flags, double *forces, int64_t f_stride, float *potentials, int64_t p_stride,
                          void *stream) {
  if (!ctx || count < 0 || (count > 0 && (!x || !forces))) return MDRT_NB_INVALID_ARGUMENT;
  if (nb_triclinic(ctx->c)) return MDRT_NB_INVALID_BOX;
  if (count > 1 && (flags & MDRT_NB_ENERGY)) return MDRT_NB_INVALID_ARGUMENT;  // one frame's energies at a time
  if (potentials && !ctx->c.pme.on) return MDRT_NB_INVALID_ARGUMENT;
  if (count == 0) return MDRT_NB_OK;
  if (!box) return MDRT_NB_INVALID_ARGUMENT;
  auto run = [&](cudaStream_t s) -> int32_t {
    for (int64_t k = 0; k < count; ++k) {
      int32_t r = nb_force_entry(ctx, x + k * x_stride, box, flags, forces + k * f_stride, s);
      if (r) return r;
      if (potentials && nb_pme_potential_grid(ctx->c, potentials + k * p_stride, s)) return MDRT_NB_CUDA_ERROR;
    }
    return MDRT_NB_OK;
  };
  // a pruning changes the context at every call: launched directly
  if (flags & MDRT_NB_PRUNE) return run((cudaStream_t)stream);
  const uint64_t args[] = {1, nb_bits(x), (uint64_t)x_stride, (uint64_t)count, nb_bits(box[0]), nb_bits(box[1]),
                           nb_bits(box[2]), flags, nb_bits(forces), (uint64_t)f_stride, nb_bits(potentials),
                           (uint64_t)p_stride};
  return nb_frames_graph(ctx, args, (int)(sizeof(args) / sizeof(args[0])), (cudaStream_t)stream, run);
}

int32_t mdrtNbParameterGradientFrames(mdrtNb *ctx, const double *x, int64_t x_stride, int64_t count,
                                      const double box[3], const double *cotangent, int64_t c_stride, int32_t mode,
                                      const float *potentials, int64_t p_stride, double *dq, double *dtable,
                                      void *stream) {
  if (!ctx || count < 0) return MDRT_NB_INVALID_ARGUMENT;
  if (count == 0) return MDRT_NB_OK;
  int32_t ready = nb_gradient_ready(ctx, x, box, cotangent, mode, potentials, dq, dtable);
  if (ready) return ready;
  auto run = [&](cudaStream_t s) -> int32_t {
    if (nb_adjoint_run(ctx->c, x, x_stride, count, box, cotangent, c_stride, mode, potentials, p_stride, dq, dtable,
                       s))
      return MDRT_NB_CUDA_ERROR;
    CK(cudaGetLastError());
    return MDRT_NB_OK;
  };
  // the energy mode's charge terms take the net charge from the host
  // charges, which the key does not hold: launched directly
  if (mode != MDRT_NB_GRAD_PRODUCT || !x || !box) return run((cudaStream_t)stream);
  const uint64_t args[] = {2, nb_bits(x), (uint64_t)x_stride, (uint64_t)count, nb_bits(box[0]), nb_bits(box[1]),
                           nb_bits(box[2]), nb_bits(cotangent), (uint64_t)c_stride, (uint64_t)mode,
                           nb_bits(potentials), (uint64_t)p_stride, nb_bits(dq), nb_bits(dtable)};
  return nb_frames_graph(ctx, args, (int)(sizeof(args) / sizeof(args[0])), (cudaStream_t)stream, run);
}

int32_t mdrtNbFrameGraphInfo(mdrtNb *ctx, int64_t *captures, int64_t *replays) {
  if (!ctx || !captures || !replays) return MDRT_NB_INVALID_ARGUMENT;
  *captures = ctx->graph_captures;
  *replays = ctx->graph_replays;
  return MDRT_NB_OK;
}

int32_t mdrtNbDisplacementStart(mdrtNb *ctx, const double *frames, int64_t count, const double box[3],
                                void *stream) {
  if (!ctx || !box || count < 0 || (count > 0 && !frames)) return MDRT_NB_INVALID_ARGUMENT;
  NbCtx &c = ctx->c;
  if (!c.built || !c.x_build) return MDRT_NB_NOT_BUILT;
  if (nb_triclinic(c)) return MDRT_NB_UNSUPPORTED;  // per-axis minimum image
  CK(cudaSetDevice(c.device));
  ctx->drift_count = -1;
  if (count == 0) {
    ctx->drift_count = 0;
    return MDRT_NB_OK;
  }
  cudaStream_t st = (cudaStream_t)stream;
  if (c.drift_cap < count) {
    nb_free(c.drift);
    if (c.h_drift) cudaFreeHost(c.h_drift);
    c.h_drift = nullptr;
    c.drift_cap = 0;
    int64_t cap = std::max<int64_t>(count, 64);
    CK(cudaMalloc(&c.drift, sizeof(unsigned long long) * cap));
    CK(cudaMallocHost(&c.h_drift, sizeof(unsigned long long) * cap));
    c.drift_cap = cap;
  }
  if (!ctx->drift_done) CK(cudaEventCreateWithFlags(&ctx->drift_done, cudaEventDisableTiming));
  CK(cudaMemsetAsync(c.drift, 0, sizeof(unsigned long long) * count, st));
  int bx = (int)std::min<int64_t>(64, std::max<int64_t>(1, (c.n + 255) / 256));
  for (int64_t f0 = 0; f0 < count; f0 += 65535) {
    int64_t nf = std::min<int64_t>(65535, count - f0);
    nb_frame_drift<<<dim3(bx, (unsigned)nf), 256, 0, st>>>(c.n, frames + f0 * 3 * c.n, c.x_build, box[0], box[1],
                                                         box[2], c.drift + f0);
  }
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(c.h_drift, c.drift, sizeof(unsigned long long) * count, cudaMemcpyDeviceToHost, st));
  CK(cudaEventRecord(ctx->drift_done, st));
  ctx->drift_count = count;
  return MDRT_NB_OK;
}

int32_t mdrtNbDisplacementResult(mdrtNb *ctx, double *out) {
  if (!ctx) return MDRT_NB_INVALID_ARGUMENT;
  NbCtx &c = ctx->c;
  if (ctx->drift_count < 0) return MDRT_NB_INVALID_ARGUMENT;  // no test started
  int64_t count = ctx->drift_count;
  ctx->drift_count = -1;
  if (count == 0) return MDRT_NB_OK;
  if (!out) return MDRT_NB_INVALID_ARGUMENT;
  CK(cudaEventSynchronize(ctx->drift_done));
  for (int64_t f = 0; f < count; ++f) {
    double d2;
    std::memcpy(&d2, &c.h_drift[f], sizeof(double));
    out[f] = std::sqrt(d2);
  }
  return MDRT_NB_OK;
}

int32_t mdrtNbDisplacement(mdrtNb *ctx, const double *frames, int64_t count, const double box[3], double *out,
                           void *stream) {
  if (!ctx || !box || count < 0 || (count > 0 && (!frames || !out))) return MDRT_NB_INVALID_ARGUMENT;
  int32_t s = mdrtNbDisplacementStart(ctx, frames, count, box, stream);
  if (s) return s;
  return mdrtNbDisplacementResult(ctx, out);
}

int32_t mdrtNbParameterGradient(mdrtNb *ctx, const double *x, const double box[3], const double *cotangent,
                                int32_t mode, double *dq, double *dtable, void *stream) {
  return mdrtNbParameterGradientPotential(ctx, x, box, cotangent, mode, nullptr, dq, dtable, stream);
}

int32_t mdrtPmePotentialGrid(mdrtNb *ctx, float *grid, void *stream) {
  if (!ctx || !grid || !ctx->c.pme.on) return MDRT_NB_INVALID_ARGUMENT;
  CK(cudaSetDevice(ctx->c.device));
  if (nb_pme_potential_grid(ctx->c, grid, (cudaStream_t)stream)) return MDRT_NB_CUDA_ERROR;
  return MDRT_NB_OK;
}

int32_t mdrtNbParameterGradientPotential(mdrtNb *ctx, const double *x, const double box[3],
                                         const double *cotangent, int32_t mode, const float *phi, double *dq,
                                         double *dtable, void *stream) {
  int32_t s = nb_gradient_ready(ctx, x, box, cotangent, mode, phi, dq, dtable);
  if (s) return s;
  if (nb_adjoint_run(ctx->c, x, 0, 1, box, cotangent, 0, mode, phi, 0, dq, dtable, (cudaStream_t)stream))
    return MDRT_NB_CUDA_ERROR;
  CK(cudaGetLastError());
  return MDRT_NB_OK;
}

int32_t mdrtNbEnergies(mdrtNb *ctx, void *stream, double *out) {
  if (!ctx || !out) return MDRT_NB_INVALID_ARGUMENT;
  NbCtx &c = ctx->c;
  cudaStream_t st = (cudaStream_t)stream;
  CK(cudaMemcpyAsync(c.h_energy, c.energy, sizeof(double) * NB_E_SLOTS, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  for (int k = 0; k < NB_E_SLOTS; ++k) out[k] = c.h_energy[k];
  return MDRT_NB_OK;
}

int32_t mdrtNbConstants(mdrtNb *ctx, const double box[3], int32_t dispersion, double *out) {
  if (!ctx || !box || !out) return MDRT_NB_INVALID_ARGUMENT;
  NbCtx &c = ctx->c;
  double sq = 0.0, net = 0.0;
  for (double v : c.h_q) {
    sq += v * v;
    net += v;
  }
  double V = box[0] * box[1] * box[2];
  out[0] = c.beta > 0 ? -c.coulomb * c.beta / std::sqrt(M_PI) * sq : 0.0;
  out[1] = c.beta > 0 ? -c.coulomb * M_PI * net * net / (2.0 * V * c.beta * c.beta) : 0.0;
  out[2] = out[3] = 0.0;
  if (dispersion) {
    int nt = c.ntypes;
    std::vector<double> cnt(nt, 0.0);
    for (int32_t t : c.h_type) cnt[t] += 1.0;
    double sum = 0.0;
    for (int a = 0; a < nt; ++a)
      for (int b = 0; b < nt; ++b) sum += cnt[a] * (cnt[b] - (a == b ? 1.0 : 0.0)) * c.h_c6[a * nt + b];
    // excluded pairs: read back the rows from the device copy
    int64_t npairs = c.n_excl_pairs;
    if (npairs > 0) {
      std::vector<int32_t> pairs(2 * npairs);
      cudaMemcpy(pairs.data(), c.excl_pairs, sizeof(int32_t) * 2 * npairs, cudaMemcpyDeviceToHost);
      for (int64_t k = 0; k < npairs; ++k)
        sum -= 2.0 * c.h_c6[c.h_type[pairs[2 * k]] * nt + c.h_type[pairs[2 * k + 1]]];
    }
    double n = (double)c.n;
    double npair = n * (n - 1.0) - 2.0 * npairs;
    double mean = npair > 0 ? sum / npair : 0.0;
    double rc = c.cutoff;
    out[2] = -2.0 * M_PI / (3.0 * V) * n * n * mean / (rc * rc * rc);
    out[3] = 2.0 * out[2];
  }
  return MDRT_NB_OK;
}

int32_t mdrtNbGroupsBuffer(mdrtNb *ctx, int32_t slot, void **pointer, int64_t *count) {
  if (!ctx || !pointer) return MDRT_NB_INVALID_ARGUMENT;
  NbCtx &c = ctx->c;
  void *p = nullptr;
  int64_t k = 0;
  switch (slot) {
    case MDRT_NB_GROUPS_ORDER: p = c.order; k = c.places_cap; break;
    case MDRT_NB_GROUPS_COUNTS: p = c.counts; k = c.groups_cap; break;
    case MDRT_NB_GROUPS_ENTRIES: p = c.slab; k = c.groups_cap * c.list_cap; break;
    case MDRT_NB_GROUPS_UNITS: p = c.units; k = c.units_cap; break;
    case MDRT_NB_GROUPS_SHIFTS: p = c.shift; k = c.places_cap; break;
    case MDRT_NB_GROUPS_INNER_ENTRIES: p = c.slab_in; k = c.slab_in ? c.slab_in_entries : 0; break;
    case MDRT_NB_GROUPS_INNER_COUNTS: p = c.counts_in; k = c.counts_in ? c.groups_cap : 0; break;
    case MDRT_NB_GROUPS_PLACED: p = c.xq; k = c.places_cap; break;
    case MDRT_NB_GROUPS_PLACE_OF: p = c.place_of; k = c.n; break;
    default: return MDRT_NB_INVALID_ARGUMENT;
  }
  *pointer = p;
  if (count) *count = k;
  return MDRT_NB_OK;
}

int32_t mdrtNbGroupsInfo(mdrtNb *ctx, int64_t *list_capacity, int64_t *builds, int64_t *grows) {
  if (!ctx) return MDRT_NB_INVALID_ARGUMENT;
  if (list_capacity) *list_capacity = ctx->c.list_cap;
  if (builds) *builds = ctx->c.builds;
  if (grows) *grows = ctx->c.grows;
  return MDRT_NB_OK;
}

int32_t mdrtNbStatus(mdrtNb *ctx, void *stream, int32_t clear, int32_t *status) {
  if (!ctx || !status) return MDRT_NB_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  int32_t v = 0;
  CK(cudaMemcpyAsync(&v, ctx->c.status, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (clear) CK(cudaMemsetAsync(ctx->c.status, 0, sizeof(int32_t), st));
  *status = v;
  return MDRT_NB_OK;
}

}  // extern "C"

// --------------------------------------------------------------------------
// FFT entries with cached plans
// --------------------------------------------------------------------------
namespace {
std::mutex g_fft_mutex;
std::map<std::tuple<int, int64_t, int64_t, int64_t, int>, cufftHandle> g_fft_plans;

cufftHandle fft_plan(int64_t k1, int64_t k2, int64_t k3, bool forward) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(g_fft_mutex);
  auto key = std::make_tuple(dev, k1, k2, k3, forward ? 1 : 0);
  auto it = g_fft_plans.find(key);
  if (it != g_fft_plans.end()) return it->second;
  cufftHandle h = 0;
  if (cufftPlan3d(&h, (int)k1, (int)k2, (int)k3, forward ? CUFFT_R2C : CUFFT_C2R) != CUFFT_SUCCESS) return 0;
  g_fft_plans[key] = h;
  return h;
}
}  // namespace

extern "C" int32_t mdrtCudaFFTForward3DF32(const float *real, float *complex_out, int64_t k1, int64_t k2,
                                           int64_t k3, void *stream) {
  if (!real || !complex_out || k1 < 1 || k2 < 1 || k3 < 1) return MDRT_NB_INVALID_ARGUMENT;
  cufftHandle h = fft_plan(k1, k2, k3, true);
  if (!h) return MDRT_NB_CUDA_ERROR;
  cufftSetStream(h, (cudaStream_t)stream);
  if (cufftExecR2C(h, (cufftReal *)real, (cufftComplex *)complex_out) != CUFFT_SUCCESS)
    return MDRT_NB_CUDA_ERROR;
  return MDRT_NB_OK;
}

extern "C" int32_t mdrtCudaFFTBackward3DF32(float *complex_in, float *real_out, int64_t k1, int64_t k2,
                                            int64_t k3, void *stream) {
  if (!real_out || !complex_in || k1 < 1 || k2 < 1 || k3 < 1) return MDRT_NB_INVALID_ARGUMENT;
  cufftHandle h = fft_plan(k1, k2, k3, false);
  if (!h) return MDRT_NB_CUDA_ERROR;
  cufftSetStream(h, (cudaStream_t)stream);
  if (cufftExecC2R(h, (cufftComplex *)complex_in, (cufftReal *)real_out) != CUFFT_SUCCESS)
    return MDRT_NB_CUDA_ERROR;
  return MDRT_NB_OK;
}

// The PME potential gathered per place, scattered to atoms in f64.
namespace {
__global__ void nb_potential_out(int64_t places, const int32_t *__restrict__ sizes,
                                 const int32_t *__restrict__ order, const float *__restrict__ pot,
                                 double *__restrict__ out) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= places || p >= sizes[NB_SIZE_PLACES]) return;
  int a = order[p];
  if (a >= 0) out[a] = pot[p];
}
}  // namespace

extern "C" int32_t mdrtPmePotential(mdrtNb *ctx, double *potential, void *stream) {
  if (!ctx || !potential) return MDRT_NB_INVALID_ARGUMENT;
  NbCtx &c = ctx->c;
  if (!c.pme.on || !c.built) return MDRT_NB_NOT_BUILT;
  cudaStream_t st = (cudaStream_t)stream;
  CK(cudaMemsetAsync(potential, 0, sizeof(double) * c.n, st));
  int blocks = (int)std::max<int64_t>(1, (c.places_cap + 255) / 256);
  nb_potential_out<<<blocks, 256, 0, st>>>(c.places_cap, c.sizes, c.order, c.pme.potential, potential);
  CK(cudaGetLastError());
  return MDRT_NB_OK;
}

extern "C" int32_t mdrtNbTimeKernels(mdrtNb *ctx, const double *x, const double box[3], int32_t iterations,
                                     void *stream, double *out) {
  if (!ctx || !x || !box || !out || iterations < 1) return MDRT_NB_INVALID_ARGUMENT;
  NbCtx &c = ctx->c;
  if (!c.built) return MDRT_NB_NOT_BUILT;
  // The launches of each stage are captured into a CUDA graph on a stream
  // of our own and the graph is timed, so that the host's launch rate does
  // not bound the numbers of short kernels.
  (void)stream;
  cudaStream_t st;
  CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  double *scratch = nullptr;
  CK(cudaMalloc(&scratch, sizeof(double) * 3 * c.n));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  auto timed = [&](auto &&launch) {
    launch();  // warm
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return -1.0;
    for (int k = 0; k < iterations; ++k) launch();
    if (cudaStreamEndCapture(st, &g) != cudaSuccess || cudaGraphInstantiate(&ge, g, 0) != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return -1.0;
    }
    cudaGraphLaunch(ge, st);
    cudaEventRecord(e0, st);
    cudaGraphLaunch(ge, st);
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaGraphExecDestroy(ge);
    cudaGraphDestroy(g);
    return (double)ms / iterations;
  };
  out[0] = timed([&] { nb_gather_frames(c, x, box, st); });
  out[1] = timed([&] { nb_pairs_run(c, box, false, st); });
  out[2] = timed([&] { nb_excluded_run(c, box, false, st); });
  out[3] = (c.pme.on && c.beta > 0) ? timed([&] { nb_pme_run(c, box, false, false, st); }) : 0.0;
  out[4] = timed([&] { nb_finish_forces(c, scratch, 0, st); });
  // the neighbor build with its present capacities (no host wait) and the
  // pruning; the lists they leave are those of x again
  out[5] = timed([&] { nb_build_launch_public(c, x, box, st); });
  nb_gather_frames(c, x, box, st);
  out[6] = c.inner_reach > 0.0 ? timed([&] { nb_prune_run(c, box, st); }) : 0.0;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  cudaFree(scratch);
  CK(cudaGetLastError());
  return MDRT_NB_OK;
}
