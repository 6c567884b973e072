// The host-side context of one system on one device: the buffers of the
// neighbor structure, the particle tables, PME plans and the scratch of the
// reductions.  Everything here is owned by the library; callers pass their
// own state (positions, forces) as plain device pointers.
#pragma once
#include <cufft.h>
#include <cstdint>
#include <vector>

#include "nb_common.cuh"

struct NbGrid {
  int Nx = 1, Ny = 1, Nz = 1;  // columns along x, y; z bins per column
  float wx = 1, wy = 1, hz = 1;  // column widths, bin height
  int ncol() const { return Nx * Ny; }
  int nbins() const { return Nx * Ny * Nz; }
};

struct NbPme {
  int K[3] = {0, 0, 0};
  int order = 4;
  bool on = false;
  cufftHandle fwd = 0, bwd = 0;
  float *grid = nullptr;        // K0*K1*K2 real grid
  float2 *spec = nullptr;       // K0*K1*(K2/2+1)
  unsigned long long *fixed = nullptr;  // deterministic spreading, K0*K1*K2
  float *moduli = nullptr;      // |b|^2 tables: K0 + K1 + K2 floats
  float *pme_force = nullptr;   // float4 per place (gather output)
  float *potential = nullptr;   // f32 per place: dE_rec/dq
  double *partials = nullptr;   // per-block energy/virial partials of the convolution
  float *adj_grid = nullptr;    // K0*K1*K2: the dipole grid V, then psi (the adjoint)
  float *influence = nullptr;   // B C per half-complex point (f32) for the sums without energy
  double infl_key[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // cell, beta, f, tilts of that table
  int conv_blocks = 0;
  size_t workspace_bytes = 0;
  float2 *fft_tw = nullptr;     // twiddles of the own transforms (nb_fft.cuh), when every K is 32, 64 or 128
  // the tiled spreading (large grids in the mixed mode): bins of
  // NB_TILE_EDGE^3 grid points, their counts (zero between spreadings) and
  // starts, and per place its bin, its rank in the bin and the places in
  // bin order
  int tile_bins[3] = {0, 0, 0};
  int32_t *tile_count = nullptr, *tile_start = nullptr, *tile_scratch = nullptr;
  int32_t *tile_bin = nullptr, *tile_rank = nullptr, *tile_sorted = nullptr;
};

// Tiles of the spreading: NB_TILE_EDGE grid points a side, in the mixed
// mode when tuned (MDIR D282: lib/Dialect/MDExec/DevicePolicy.cpp:105-124,
// bins of 8 points; not in the deterministic mode, as MDIR).
#define NB_TILE_EDGE 8

struct NbCtx {
  int device = 0;
  int64_t n = 0;
  // particle tables (atom order)
  float *q = nullptr;
  int32_t *type = nullptr;
  int32_t ntypes = 0;
  float2 *lj = nullptr;  // (c6, c12) per type pair, c6 = 4 eps sig^6, c12 = 4 eps sig^12
  float2 *ljf = nullptr;  // per type (sqrt c6, sqrt c12) when the table factorizes
  bool lj_geom = false;   // c6_ab = f_a f_b and c12_ab = g_a g_b for every pair of types
  std::vector<double> h_q;     // f64 charges for the host constants
  std::vector<double> h_c6;    // f64 c6 = 4 eps sig^6 per type pair
  std::vector<int32_t> h_type;
  std::vector<float2> h_lj;
  float2 *sigeps = nullptr;    // (sigma, epsilon) per type pair, for the parameter gradient
  int32_t *lj_on = nullptr;    // per type: 1 when an epsilon of its row is not 0 (device, 32 types)
  uint32_t lj_mask = 0;        // the same, a bit per type
  // exclusions: ragged rows (atom order) and the list of pairs i < j
  int32_t *excl_off = nullptr, *excl = nullptr;
  int32_t *excl_pairs = nullptr;
  int64_t n_excl_pairs = 0;
  // interaction parameters
  double cutoff = 1.0, reach = 1.1, beta = 0.0, coulomb = 138.935457644;
  int coulomb_shift = 0, lj_switch = 0;
  double switch_distance = 0.0;
  bool deterministic = false;
  // neighbor structure
  NbGrid grid;
  double box_built[3] = {0, 0, 0};
  // The tilts (bx, cx, cy) of a triclinic cell whose diagonal is the box
  // (mdrtNbBuildTriclinic / mdrtNbForceTriclinic); 0 for an orthorhombic one.
  double tilt[3] = {0, 0, 0};
  double tilt_built[3] = {0, 0, 0};
  int64_t groups_cap = 0, places_cap = 0, bins_cap = 0, cols_cap = 0;
  int64_t list_cap = 0;    // C: entries per group
  int64_t units_cap = 0;
  int32_t *order = nullptr, *place_of = nullptr;
  char4 *shift = nullptr;  // per place
  float4 *xw = nullptr;    // per place, f32 wrapped at the build
  float4 *box_lo = nullptr, *box_hi = nullptr;  // per group
  int32_t *group_start = nullptr;  // per column + 1
  int32_t *group_col = nullptr;    // per group
  int2 *slab = nullptr;            // groups_cap * list_cap entries
  int32_t *counts = nullptr;       // per group
  int32_t *unit_n = nullptr, *unit_start = nullptr;  // per group (+1)
  int2 *units = nullptr;           // (group, ordinal)
  int32_t *sizes = nullptr;        // NB_SIZE_COUNT ints on the device
  int32_t *h_sizes = nullptr;      // pinned mirror
  int32_t *status = nullptr;       // device status word
  // build scratch
  int32_t *key = nullptr, *bin_count = nullptr, *bin_start = nullptr, *bin_fill = nullptr;
  int32_t *sorted = nullptr, *col_groups = nullptr, *scan_scratch = nullptr;
  float4 *atom_xw = nullptr;
  char4 *atom_shift = nullptr;
  // per-step frames and accumulators (place order)
  float4 *xq = nullptr;
  float4 *xq_lo = nullptr;               // the f32 residual of each frame (deterministic mode: split frames)
  int32_t *typ_p = nullptr;
  float4 *acc = nullptr;                 // pair + excluded forces, f32 atomics
  unsigned long long *acc_fixed = nullptr;  // 3 per place, deterministic mode
  double *unit_partials = nullptr;       // 8 doubles per unit
  double *excl_partials = nullptr;       // 8 doubles per block of the excluded kernel
  double *energy = nullptr;              // device results: see NbEnergySlot
  double *h_energy = nullptr;            // pinned mirror
  NbPme pme;
  bool built = false;
  int64_t builds = 0, grows = 0;
  // the inner list of the dual list (MDIR D114): the outer lists pruned to
  // `inner_reach` at the positions of the last pruning; same layout, same
  // capacity per group.  inner_reach = 0: one list.
  double inner_reach = 0.0;
  bool inner_valid = false;
  int64_t inner_key = -1;  // the outer capacities the inner buffers were sized for
  int2 *slab_in = nullptr;
  int64_t slab_in_entries = 0;  // the allocation of slab_in (the search stages in it)
  int32_t *counts_in = nullptr;
  int32_t *unit_n_in = nullptr, *unit_start_in = nullptr;
  int2 *units_in = nullptr;
  int32_t *sizes_in = nullptr;  // NB_SIZE_UNITS of the inner list (device)
  int64_t prunes = 0;
  // tuning (mdrtNbSetTuning): blocks of 8 warps per SM of the pair kernel
  int pair_blocks_per_sm = 4;
  int pair_sms = 0;  // SMs the persistent pair grid spans (0: all); the rest are left to PME
  int fused_prune = 0;  // the MD step's pruning in the pair kernel: 0 by group count, 1 always, 2 never
  int pme_spread = 0;  // the spreading: 0 (the default) and 1, global atomics; 2, tiles (mixed mode)
  int pme_fft = 0;  // the PME transforms: 0, the own three-kernel convolution where the grid allows; 1, cuFFT
  int staging_depth = 1;  // the pair kernel's force forms: 1, a unit's entries read as it starts; 2, during the unit before
  int frame_graphs = 1;  // the frames entries replay their launches as CUDA graphs (1) or launch them (0)
  int32_t *one = nullptr;  // a device 1: the gate of a pruning a force call asks for (MDRT_NB_PRUNE)
  // parameter gradient scratch (mdrtNbParameterGradient), allocated at the first call
  float4 *adj_g = nullptr;        // per place: the cotangent on the forces (f32)
  double *adj_q = nullptr;        // per place: the charge gradient, kept zero between calls
  double *adj_types = nullptr;    // per block of the adjoint kernel: 2 ntypes^2 partials
  int adj_width = 0;              // the 2 ntypes^2 adj_types was sized for
  int64_t adj_places = 0;         // places_cap the per-place arrays were sized for
  int adj_blocks = 0;
  // the outer lists of a build without a pruned reach with each group's
  // entries of a partner with Lennard-Jones terms first (nb_lj_partition_run):
  // their count per group, for the build `lj_part_build` and the types of
  // `lj_part_mask`; the adjoint's rounds after them skip their LJ terms
  int32_t *counts_lj = nullptr;
  int64_t counts_lj_cap = 0;
  int64_t lj_part_build = -1;
  uint32_t lj_part_mask = 0;
  // the columns and bins the buffers are planned for (one grid, or the
  // frames of a batch laid end to end)
  int64_t plan_cols = 0, plan_bins = 0;
  // the f64 positions of the last build (atom order) and the per-frame
  // displacement maxima of mdrtNbDisplacement
  double *x_build = nullptr;
  unsigned long long *drift = nullptr;
  unsigned long long *h_drift = nullptr;  // pinned mirror
  int64_t drift_cap = 0;
};

// Energy / virial slots of ctx->energy (f64, device).
enum NbEnergySlot {
  NB_E_LJ = 0,
  NB_E_COUL = 1,
  NB_E_EXCL = 2,
  NB_E_REC = 3,
  NB_W_PAIR = 4,   // 6 entries: xx yy zz xy xz yz (pairs + excluded)
  NB_W_REC = 10,   // 6 entries
  NB_E_SLOTS = 16
};

// The launches of one frames call kept as a CUDA graph (nb_api.cu): the
// key is the call's arguments followed by the bytes of the context it ran
// in; exec is null for a key seen once and not yet captured.
struct NbFrameGraph {
  std::vector<unsigned char> key;
  cudaGraphExec_t exec = nullptr;
  uint64_t used = 0;
};

// The opaque handle of the C ABI.
struct mdrtNb {
  NbCtx c;
  std::vector<NbFrameGraph> graphs;
  uint64_t graph_clock = 0;
  cudaStream_t capture = nullptr;  // the frames graphs are captured on this stream
  int64_t graph_captures = 0, graph_replays = 0;
  // a started displacement test (mdrtNbDisplacementStart): the event after
  // the copy of its result and its frames (-1 when none is pending); kept
  // out of NbCtx, whose bytes key the frames graphs
  cudaEvent_t drift_done = nullptr;
  int64_t drift_count = -1;
};

// One frame of a batch, as the kernels read it: the cell, its grid of
// columns and bins and where they sit among the batch's, the widened
// reach, and its PME grid.
struct NbFrameDev {
  double L0, L1, L2;
  float Lf0, Lf1, Lf2;
  float inv_wx, inv_wy, inv_hz;
  float wx, wy;
  int Nx, Ny, Nz;
  int bin0, col0, ncol;
  float R2f, Rbox;
  int K0, K1, K2, mod0;
  long long grid0, spec0;
  double pref, pi2_beta2;  // the influence function: f/(pi V), pi^2/beta^2
  int atom0, natoms;
};

// Many independent systems (frames) evaluated together: the atoms of all
// frames are numbered one after the other, and one NbCtx holds the places,
// groups, lists, units and accumulators of all of them.  The grids of the
// frames lie end to end (bins and columns), so that every stage of the
// build, the pair kernel and PME is one launch over all frames; a group,
// a column and an atom know their frame.
struct mdrtNbBatch {
  mdrtNb *nb = nullptr;  // the shared context, n = all atoms
  int32_t frames = 0;
  std::vector<int64_t> atom0;  // frames + 1
  std::vector<NbFrameDev> h_frames;
  NbFrameDev *frames_dev = nullptr;
  int32_t *atom_frame = nullptr;  // per atom
  int32_t *atom_col = nullptr;    // per atom: its column at the build
  int32_t *col_frame = nullptr;   // per column
  int32_t *group_frame = nullptr; // per group
  float4 *group_L = nullptr;      // per group: the frame's cell
  int64_t groups_alloc = 0, cols_alloc = 0;
  int32_t *frame_units = nullptr; // per frame: first unit, one past the last
  int2 *search_scratch = nullptr; // the search's chunks with four warps a group (groups_cap x list_cap)
  int64_t search_scratch_entries = 0;
  std::vector<double> h_boxes;    // frames x 3 of the last build
  // excluded pairs: blocks of 256 pairs that never straddle two frames
  int32_t *excl_blk_frame = nullptr, *excl_blk_first = nullptr, *excl_frame_end = nullptr;
  std::vector<int32_t> h_excl_blk0;  // frames + 1
  int excl_blocks = 0;
  double *excl_part = nullptr;
  // PME: frames sorted by grid shape; one batched cuFFT plan pair a shape
  int order = 4;
  bool pme = false;
  struct Shape {
    int K[3];
    int count;
    long long grid0, spec0;
    cufftHandle fwd, bwd;
  };
  std::vector<Shape> shapes;
  long long grid_points = 0;  // real grid points of all frames
  int32_t *conv_blk_frame = nullptr;
  std::vector<int32_t> h_conv_blk0;  // frames + 1
  int conv_blocks = 0;
  double *conv_part = nullptr;
  int32_t *d_excl_blk0 = nullptr, *d_conv_blk0 = nullptr;
  // energies: frames x NB_E_SLOTS (device) and a pinned mirror
  double *frame_energy = nullptr, *h_frame_energy = nullptr;
  int search_warps = 4;  // tuning: warps a group of the search (1 or 4)
  // the force evaluation as a CUDA graph
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;
  const double *gx = nullptr;
  double *gf = nullptr;
  uint32_t gflags = 0;
  int64_t gkey = -1;
};

// Launchers implemented in the .cu files.
int nb_build_run(NbCtx &c, const double *x, const double box[3], cudaStream_t s);
// One build's launches with the current capacities, no host wait (a graph
// body); overflow is left in c.sizes.
void nb_build_launch_public(NbCtx &c, const double *x, const double box[3], cudaStream_t s);
// The pruning of the outer lists into the inner ones at the current frames
// xq (gathered by the caller), and the inner units; no host wait.
void nb_prune_run(NbCtx &c, const double box[3], cudaStream_t s);
// The same pruning as two launches that do nothing unless *gate (device) is
// set: the inner lists with the positions of the pruning copied to x_prune,
// then the inner units in one block, counting the pruning in *prunes.  The
// per-step pruning of the MD step, which needs no conditional node.
void nb_prune_gated(NbCtx &c, const double box[3], const int *gate, const double *x, double *x_prune,
                    double *prunes, int32_t *unit_counter, cudaStream_t s);
// Allocates the inner lists to the outer capacities (host, between launches).
int nb_reserve_inner(NbCtx &c);
// Grows the list capacity for lists of up to `longest` entries (+25%), as
// the count of a build that overflowed asks (host, between launches).
int nb_grow_lists(NbCtx &c, int64_t longest);
// The same growth keeping the lists in force: their entries and units are
// copied into the larger buffers, so nothing needs a build (host wait on s).
int nb_grow_lists_keep(NbCtx &c, int64_t longest, cudaStream_t s);
// Lists longer than this fraction of the capacity are grown ahead, before a
// rebuild inside the step graphs overflows.
#define NB_GROW_AHEAD 0.85
// With `cot` (f64 [n,3], atom order), its f32 copy in place order goes to
// c.adj_g as well (the adjoint's cotangent).
void nb_gather_frames(NbCtx &c, const double *x, const double box[3], cudaStream_t s,
                      const double *cot = nullptr);
// With `halt` (device), nothing when *halt is set (the MD step's stop).
// With `skip` (device), nothing when *skip is set (a pruning step whose
// pairs nb_prune_pairs_run computed).
// With `update_after`, the kernel lets the chained launch after it (the MD
// step's update) start beside it once its persistent blocks are resident;
// kept off where pair launches follow one another.
void nb_pairs_run(NbCtx &c, const double box[3], bool energy, cudaStream_t s, const int *halt = nullptr,
                  const int *skip = nullptr, bool update_after = false);
// The pruning of a pruning step with the pairs of its fresh inner lists in
// one kernel (MDIR D284), when *gate (device) is set: the same inner lists
// and claimed units as nb_prune_gated, the forces of the pairs added.
// Forces only, outside the deterministic mode.
void nb_prune_pairs_run(NbCtx &c, const double box[3], const int *gate, const double *x, double *x_prune,
                        double *prunes, int32_t *unit_counter, cudaStream_t s, const int *halt);
// Whether the MD step prunes in its pair kernel: the tuning (fused_prune),
// by default from NB_FUSED_PRUNE_GROUPS groups of the last build on (MDIR's
// threshold, DevicePolicy.cpp:70-99); never in the deterministic mode or
// with lists too long for the kernel's shared-memory staging.
bool nb_fused_prune(const NbCtx &c);
// The PME convolution runs on the own three kernels (nb_fft.cuh): every
// grid dimension 32, 64 or 128 and cuFFT not asked for.
bool nb_fft_own(const NbCtx &c);
// The spreading takes tiles (large grids in the mixed mode, or as tuned).
bool nb_pme_tiled(const NbCtx &c);
#define NB_FUSED_PRUNE_GROUPS 4096
#define NB_FUSED_STAGE_MAX (160 * 1024)
void nb_excluded_run(NbCtx &c, const double box[3], bool energy, cudaStream_t s);
// The correction over a given list of pairs (i < j), forces only.
void nb_excluded_list_run(NbCtx &c, const double box[3], const int32_t *pairs, int64_t npairs,
                          cudaStream_t s);
void nb_finish_forces(NbCtx &c, double *forces, int accumulate, cudaStream_t s);
void nb_reduce_energy(NbCtx &c, bool pairs, bool excluded, cudaStream_t s);
int nb_pme_setup(NbCtx &c, int k0, int k1, int k2, int order);
void nb_pme_release(NbCtx &c);
int nb_pme_run(NbCtx &c, const double box[3], bool energy, bool potential, cudaStream_t s);
// The parameter gradient (mdrtNbParameterGradient) summed over `count`
// frames (x + k x_stride; cotangent + k c_stride; phi + k p_stride when phi
// is given).  mode 0: the product sum_k g_k . dF_k/dtheta for the cotangent
// g (f64 [n,3], atom order); mode 1: dE/dtheta.  Adds the charge gradient to
// dq (f64 [n], atom order) and the type-pair gradient to dtable (f64,
// ntypes^2 sigma entries then ntypes^2 epsilon entries), each reduced once
// at the end of the call.  Needs the adjoint scratch (nb_adjoint_reserve).
int nb_adjoint_reserve(NbCtx &c);
// After a build (host, stream s): the stable partition of each group's
// entries by whether the partner's type has LJ terms, when the lists are
// the ones the kernels walk (no pruned reach) and fit the kernel's staging.
int nb_lj_partition_run(NbCtx &c, cudaStream_t s);
int nb_adjoint_run(NbCtx &c, const double *x, int64_t x_stride, int64_t count, const double box[3],
                   const double *cotangent, int64_t c_stride, int mode, const float *phi, int64_t p_stride,
                   double *dq, double *dtable, cudaStream_t s);
// The reciprocal part of the charge gradient, added per place into c.adj_q.
int nb_pme_potential_grid(NbCtx &c, float *out, cudaStream_t s);
// With phi (a potential grid kept from the force evaluation at the same
// frames and charges), the reciprocal forward is not run again.
int nb_pme_adjoint_run(NbCtx &c, const double box[3], int mode, cudaStream_t s, const float *phi = nullptr);

// The MD step's reciprocal chain when the update gathers (order 4): the
// frames spread into qgrid (through qfixed, empty, in the deterministic
// mode) -> spec -> phi, on the integrator's own buffers.
int nb_pme_md_chain(NbCtx &c, const double box[3], float *qgrid, unsigned long long *qfixed, float2 *spec,
                    float *phi, const float *influence, const int *halt, cudaStream_t s);
int nb_pme_influence(NbCtx &c, const double box[3], float *influence, cudaStream_t s);

// The batch (mdrtNbBatch): the build of all frames (grows and builds again
// until every list fits; host wait), the frames of the places, the pair
// kernel, the excluded pairs, PME, and the per-frame energy sums.
int nb_batch_build_run(mdrtNbBatch &b, const double *x, cudaStream_t s);
void nb_batch_gather_frames(mdrtNbBatch &b, const double *x, cudaStream_t s);
void nb_batch_pairs_run(mdrtNbBatch &b, bool energy, cudaStream_t s);
void nb_batch_excluded_run(mdrtNbBatch &b, bool energy, cudaStream_t s);
int nb_batch_pme_setup(mdrtNbBatch &b, const int32_t *grids, int order);
void nb_batch_pme_release(mdrtNbBatch &b);
int nb_batch_pme_run(mdrtNbBatch &b, bool energy, cudaStream_t s);
void nb_batch_energy_sums(mdrtNbBatch &b, bool pairs, bool excluded, bool pme, cudaStream_t s);

// The f32 cell of a context's box and tilts.
inline NbCell nb_cell(const NbCtx &c, const double box[3]) {
  NbCell H;
  H.ax = (float)box[0];
  H.by = (float)box[1];
  H.cz = (float)box[2];
  H.bx = (float)c.tilt[0];
  H.cx = (float)c.tilt[1];
  H.cy = (float)c.tilt[2];
  return H;
}
inline bool nb_triclinic(const NbCtx &c) { return c.tilt[0] != 0.0 || c.tilt[1] != 0.0 || c.tilt[2] != 0.0; }
