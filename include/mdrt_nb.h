/* mdrt_nb.h: C ABI of the B200 short-range nonbonded + PME term.
 *
 * A drop-in for the part of MDIR's device runtime that builds the groups of
 * neighbors, runs the pair loop of Lennard-Jones + Ewald real space, and the
 * PME spreading / FFT / gathering.  In MDIR these are emitted kernels called
 * through the MLIR GPU runtime ABI plus `mdrt*` entries of
 * runtime/mdrt_cuda.c; here they are one shared library with plain pointers
 * and sizes (no CUDA or torch types in the signatures: a stream is passed as
 * `void *`, i.e. a cudaStream_t, NULL for the default stream).
 *
 * Units: nm, ps, kJ/mol, e.  Device arrays are marked "device"; everything
 * else is host memory.  Every entry returns an mdrtNbStatus; none aborts.
 * A context is not thread-safe; all work goes to the caller's stream.
 */
#ifndef MDRT_NB_H
#define MDRT_NB_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MDRT_NB_ABI_VERSION 2

typedef struct mdrtNb mdrtNb;

/* Status codes.  MDIR aborts on driver errors (runtime/mdrt_cuda.c:49-71)
 * and stops a run through a handler (mdrt_cuda.c:2560-2577); this library
 * returns them instead. */
enum mdrtNbStatus {
  MDRT_NB_OK = 0,
  MDRT_NB_GROW = 1,             /* a buffer was too small; grown, call again */
  MDRT_NB_NAN_POSITION = 2,     /* positions not finite or far outside the cell */
  MDRT_NB_INVALID_BOX = 3,      /* reach >= 0.999 of the least edge, or a bad edge */
  MDRT_NB_CUDA_ERROR = 4,
  MDRT_NB_TIMEOUT = 5,
  MDRT_NB_INVALID_ARGUMENT = 6,
  MDRT_NB_UNSUPPORTED = 7,
  MDRT_NB_OVERFLOW = 8,         /* fixed-point accumulator out of range */
  MDRT_NB_NOT_BUILT = 9         /* a force call before the first build */
};

/* Flags of mdrtNbForce. */
enum mdrtNbFlags {
  MDRT_NB_ENERGY = 1u,       /* energies and virial (f64, fixed order) */
  MDRT_NB_ACCUMULATE = 2u,   /* add into `forces` instead of overwriting */
  MDRT_NB_POTENTIAL = 4u,    /* also gather dE_rec/dq (mdrtPmePotential) */
  MDRT_NB_NO_PAIRS = 8u,     /* skip the pair term */
  MDRT_NB_NO_PME = 16u,      /* skip the reciprocal sum */
  MDRT_NB_NO_EXCLUDED = 32u, /* skip the excluded-pair correction */
  MDRT_NB_GRAPH = 64u,       /* mdrtNbBatchForce: replay the launches as a CUDA graph */
  /* prune the dual list at x first, as mdrtNbPrune does; for forces
   * without energies outside the deterministic mode the pruning and the
   * pairs of the fresh inner lists run as one kernel (MDIR D284) */
  MDRT_NB_PRUNE = 128u
};

/* Slots of the energies of mdrtNbEnergies (f64). */
enum mdrtNbEnergySlot {
  MDRT_NB_E_LJ = 0,
  MDRT_NB_E_COULOMB = 1,     /* Ewald direct */
  MDRT_NB_E_EXCLUDED = 2,    /* -f q q erf(beta r)/r over excluded pairs */
  MDRT_NB_E_RECIPROCAL = 3,
  MDRT_NB_W_PAIR = 4,        /* 6: xx yy zz xy xz yz of pairs + excluded */
  MDRT_NB_W_RECIPROCAL = 10, /* 6 */
  MDRT_NB_E_COUNT = 16
};

/* Slots of the build's sizes (MDIR's sizes[5] of
 * mdrt_gpu_build_neighbors_groups, GroupsBuild.cpp:2517-2547, plus three). */
enum mdrtNbSizeSlot {
  MDRT_NB_SIZE_PLACES = 0,
  MDRT_NB_SIZE_LONGEST = 1,
  MDRT_NB_SIZE_UNITS = 2,   /* MDIR: blocks; here units of 64 entries */
  MDRT_NB_SIZE_EXCL_WIDE = 3,
  MDRT_NB_SIZE_NAN = 4,
  MDRT_NB_SIZE_OVERFLOW = 5,
  MDRT_NB_SIZE_GROUPS = 6,
  MDRT_NB_SIZE_ENTRIES = 7,
  MDRT_NB_SIZE_COUNT = 8
};

/* Buffer slots of mdrtNbGroupsBuffer, after MDIR's stable slot table
 * (include/mdir/Runtime/GroupsABI.h:10-44). */
enum mdrtNbGroupsSlot {
  MDRT_NB_GROUPS_ORDER = 0,    /* int32 [places]: atom at a place, -1 empty */
  MDRT_NB_GROUPS_COUNTS = 1,   /* int32 [groups]: entries of each list */
  MDRT_NB_GROUPS_ENTRIES = 2,  /* int32x2 [groups * capacity]: (place, mask | image << 16) */
  MDRT_NB_GROUPS_UNITS = 4,    /* int32x2 [units]: (group, ordinal) */
  MDRT_NB_GROUPS_SHIFTS = 6,   /* int8x4 [places]: whole cells S of each place */
  /* the pruned (inner) lists of a dual list, valid after a pruning: the
   * entries of the outer lists with the members within the pruned reach, by
   * member count (more than NB_SPARSE_BITS = 5 first, then 1, 2, ..., 5), in
   * the outer order within a count (lists of more than 25,600 entries, past
   * the pruning's shared-memory staging, keep the outer order); none
   * without a dual list */
  MDRT_NB_GROUPS_INNER_ENTRIES = 7, /* int32x2 [groups * capacity] */
  MDRT_NB_GROUPS_INNER_COUNTS = 9,  /* int32 [groups] */
  MDRT_NB_GROUPS_PLACED = 15,  /* float32x4 [places]: frames (x + (S - 1/2) L, q), centred on the cell */
  MDRT_NB_GROUPS_PLACE_OF = 16 /* int32 [particles]: place of each atom, -1 none */
};

/* Library and ABI version (MDRT_NB_ABI_VERSION). */
int32_t mdrtNbVersion(void);
/* A message for a status code (static storage). */
const char *mdrtNbStatusString(int32_t status);

/* A context for `particles` atoms on CUDA device `device`.
 * MDIR: mdrtGroupsCreate(places, blocks), runtime/mdrt_cuda.c:3087. */
int32_t mdrtNbCreate(mdrtNb **out, int32_t device, int64_t particles);
int32_t mdrtNbDestroy(mdrtNb *ctx);

/* Charges (e) and LJ types of each atom, and the sigma / epsilon of each
 * type pair (ntypes x ntypes, nm and kJ/mol), all host arrays.
 * MDIR: the fields and the folded type-pair table (D96) of the pair loop,
 * lib/Driver/TermNonbonded.cpp:1423-1557. */
int32_t mdrtNbSetParticles(mdrtNb *ctx, const double *charges, const int32_t *types,
                           int32_t ntypes, const double *sigma, const double *epsilon);

/* Excluded pairs as ragged rows in atom order, both directions:
 * offsets[particles + 1], partners[offsets[particles]] (host).
 * MDIR: the `excluded` incidence rows of the build,
 * GroupsBuild.cpp:2517-2547 (include/mdir/Conversion/RaggedRows.h). */
int32_t mdrtNbSetExclusions(mdrtNb *ctx, const int32_t *offsets, const int32_t *partners);

/* Cutoff r_c, reach R (r_c + skin), Ewald beta (0: no Coulomb direct sum),
 * Coulomb constant f, the direct-sum shift erfc(beta r_c)/r_c (0/1), and
 * the switch of the LJ potential from switch_distance rs to r_c: 0 none;
 * 1 the cubic in r^2, S = (1 - y)^2 (1 + 2y), y = (r^2 - rs^2)/(r_c^2 - rs^2)
 * (MDIR's SQUARED_DISTANCE_SWITCH modifier, TermLennardJones.cpp:72-95);
 * 2 the quintic in r, S = 1 - 10t^3 + 15t^4 - 6t^5, t = (r - rs)/(r_c - rs)
 * (the potential switch of MDIR's md dialect, lib/Dialect/MD/Transforms/
 * ExpandTruncation.cpp:19-46).
 * MDIR: TermNonbonded.cpp:378-470 and TermLennardJones.cpp:26-80. */
int32_t mdrtNbSetInteraction(mdrtNb *ctx, double cutoff, double reach, double beta, double coulomb,
                             int32_t coulomb_shift, int32_t lj_switch, double switch_distance);

/* The dual list: the lists built at the reach R are pruned to
 * pruned_distance (r_c <= it < R; 0 or R: one list), and the force term
 * reads the pruned ones.  MDIR: `pruned_distance` of [energy] (D114,
 * docs/neighbor-groups.md, Section 6.2). */
int32_t mdrtNbSetPrunedReach(mdrtNb *ctx, double pruned_distance);

/* Prunes the lists at device positions x (after a build whose lists are
 * valid for x): inner mask = outer mask and r <= pruned_distance, entries
 * with no bit left dropped.  MDIR: emitGroupsPrune,
 * lib/Conversion/MDExecToGPU/MDExecToGPU.cpp:9588. */
int32_t mdrtNbPrune(mdrtNb *ctx, const double *x, const double box[3], void *stream);

/* Launch-shape tuning of the kernels (the autotuner's knobs; results do not
 * depend on them): MDRT_NB_TUNE_PAIR_BLOCKS_PER_SM, the resident blocks of 8
 * warps per SM of the pair kernel (1-4; fewer leave room for the PME
 * kernels beside it).  Returns MDRT_NB_INVALID_ARGUMENT for an unknown key
 * or value.  No MDIR counterpart: MDIR fixes these in its emitters
 * (lib/Dialect/MDExec/DevicePolicy.cpp:72-99). */
enum mdrtNbTuneKey {
  MDRT_NB_TUNE_PAIR_BLOCKS_PER_SM = 0,
  MDRT_NB_TUNE_SEARCH_WARPS = 1,  /* batches only */
  MDRT_NB_TUNE_PAIR_SMS = 2,      /* SMs the pair grid spans (0: all); the others stay free for PME */
  /* the MD step's pruning of the dual list in its pair kernel (MDIR D284,
   * lib/Dialect/MDExec/DevicePolicy.cpp:70-99): 0 from 4096 groups on (the
   * default), 1 always, 2 never; never in the deterministic mode */
  MDRT_NB_TUNE_FUSED_PRUNE = 3,
  /* the pair kernel's staging depth: 1, a unit's entries are read as the
   * unit starts; 2, the next unit's entries are in flight during a unit */
  MDRT_NB_TUNE_STAGING_DEPTH = 4,
  /* the PME transforms: 0, the library's own three-kernel convolution when
   * every grid dimension is 32, 64 or 128 (the default), cuFFT otherwise;
   * 1, cuFFT always (MDIR's cuFFT path, runtime/mdrt_cuda.c:2942-2990) */
  MDRT_NB_TUNE_PME_FFT = 5,
  /* the PME spreading: 0 (the default) and 1, global atomics; 2, through
   * shared-memory tiles of 8^3 grid points in the mixed mode (MDIR D282,
   * lib/Dialect/MDExec/DevicePolicy.cpp:105-124, which tiles grids of
   * 500,000 points by default on its devices; on the B200 the global atomics
   * measured faster at 224^3).  The deterministic mode spreads in fixed
   * point with global atomics. */
  MDRT_NB_TUNE_PME_SPREAD = 6,
  /* the frames entries (mdrtNbForceFrames, mdrtNbParameterGradientFrames):
   * 1, their launches kept and replayed as CUDA graphs (the default); 0,
   * launched on each call */
  MDRT_NB_TUNE_FRAME_GRAPHS = 7
};
int32_t mdrtNbSetTuning(mdrtNb *ctx, int32_t key, int32_t value);

/* Deterministic mode: 64-bit fixed-point force accumulation (2^32 per
 * kJ/mol/nm) and PME spreading (2^40 per e); bitwise reproducible.
 * MDIR: deterministic = true (D70, D84; docs/pme.md, Section 3). */
int32_t mdrtNbSetDeterministic(mdrtNb *ctx, int32_t on);

/* The PME grid k1 x k2 x k3 and the spline order (4, 5, 6 or 8).
 * MDIR: the PME plan and cuFFT plans, mdrtRetainFFTPlan, mdrt_cuda.c:2765. */
int32_t mdrtPmeSetup(mdrtNb *ctx, int32_t k1, int32_t k2, int32_t k3, int32_t order);

/* The neighbor build from device positions x (f64 [n, 3], unwrapped) in the
 * orthorhombic cell box[3].  Grows its buffers and builds again until every
 * list fits (count-then-grow), then writes MDRT_NB_SIZE_COUNT sizes to
 * sizes_out (host, may be NULL).  Returns MDRT_NB_NAN_POSITION (after a
 * complete build that leaves those atoms out) if any position is not finite.
 * MDIR: mdrt_gpu_build_neighbors_groups(x, box, reach, excluded, order,
 * placeOf, entries, masks, counts, units, ordinals, shifts, sizes),
 * lib/Conversion/MDExecKernels/GroupsBuild.cpp:2515-2550, with
 * mdrtGroupsGrow (mdrt_cuda.c:3185) and the retry loop of
 * lib/Conversion/MDExecToGPU/MDExecToGPU.cpp:10107-10175. */
int32_t mdrtNbBuild(mdrtNb *ctx, const double *x, int64_t n, const double box[3], double reach,
                    void *stream, int32_t *sizes_out);

/* The force term at device positions x (f64 [n, 3]): writes (or adds, with
 * MDRT_NB_ACCUMULATE) the forces of the pairs, the excluded-pair correction
 * and PME to `forces` (device f64 [n, 3]).  Needs a build whose lists are
 * still valid for x.  Asynchronous on `stream`.
 * MDIR: the emitted pair loop (TraversePairs.cpp:85), the excluded tuple
 * loop (TermNonbonded.cpp:1615) and the reciprocal stages
 * (MDExecToGPU/DevicePME.cpp:38-75). */
int32_t mdrtNbForce(mdrtNb *ctx, const double *x, const double box[3], uint32_t flags,
                    double *forces, void *stream);

/* The build and the force term in a triclinic cell: cell = (ax, by, cz,
 * bx, cx, cy), the rows a = (ax, 0, 0), b = (bx, by, 0), c = (cx, cy, cz)
 * of a lower-triangular H in the reduced form |bx|, |cx| <= ax/2,
 * |cy| <= by/2 (else MDRT_NB_INVALID_BOX; also a reach of 0.999 of the
 * least of ax, by, cz or more).  Positions are wrapped into the brick
 * [0, ax) x [0, by) x [0, cz) along c, then b, then a; an entry's image is a
 * lattice vector n (five bits a component), applied as n H; the reach is
 * widened by 3e-6 of the sum of the diagonal and the tilts' magnitudes.
 * The lists hold every image within the reach once (several images of a
 * pair when the reach exceeds half the cell).  A context built in a
 * triclinic cell takes its forces from mdrtNbForceTriclinic with the same
 * cell (mdrtNbForce refuses it); the pruning, energies, constants and
 * mdrtPmePotential work as in an orthorhombic cell (box = the diagonal).
 * PME spreads and gathers on the fractional coordinates f = x H^-1 with the
 * wave vectors m = H^-1 k (docs/pme.md, Section 1; V = ax by cz).  The
 * parameter gradient and the displacement test run in orthorhombic cells
 * only (MDRT_NB_UNSUPPORTED); the MD step and batches build orthorhombic
 * cells.
 * MDIR: mdrt_gpu_build_neighbors_groups_triclinic(x, vector<6xf64>, ...)
 * (GroupsBuild.cpp:248-345, docs/neighbor-groups.md Section 5.1, D126);
 * its lists are checked by test/Runtime/neighbors-groups-triclinic-gpu.mlir. */
int32_t mdrtNbBuildTriclinic(mdrtNb *ctx, const double *x, int64_t n, const double cell[6], double reach,
                             void *stream, int32_t *sizes_out);
int32_t mdrtNbForceTriclinic(mdrtNb *ctx, const double *x, const double cell[6], uint32_t flags,
                             double *forces, void *stream);

/* Copies the energies and virials of the last MDRT_NB_ENERGY evaluation
 * (MDRT_NB_E_COUNT f64) to out (host); waits for `stream`.
 * MDIR: the seven f64 numbers per sum of docs/pme.md, Section 3, and
 * TraverseHost::finishSums (include/mdir/Conversion/TraversePairs.h:130-137). */
int32_t mdrtNbEnergies(mdrtNb *ctx, void *stream, double *out);

/* Host constants of the Ewald sum and the LJ tail in the cell box[3]:
 * out[0] self -f beta/sqrt(pi) sum q^2, out[1] background
 * -f pi Q^2/(2 V beta^2), out[2] dispersion correction -2 pi N^2 <C6>/(3 V rc^3)
 * (0 unless `dispersion`), out[3] its virial per diagonal entry (2 E_disp).
 * MDIR: TermNonbonded.cpp:601-637 and 651-668. */
int32_t mdrtNbConstants(mdrtNb *ctx, const double box[3], int32_t dispersion, double *out);

/* dE_rec/dq_i of the last evaluation made with MDRT_NB_POTENTIAL, to
 * potential (device f64 [n]).  MDIR: the PME potential stage (D231). */
int32_t mdrtPmePotential(mdrtNb *ctx, double *potential, void *stream);

/* The largest displacement (nm, minimum image) of each of `count` frames
 * (device f64 [count, n, 3]) from the positions of the last build, to out
 * (host f64 [count]); +inf for a frame with a coordinate that is not
 * finite.  The lists of the build serve a frame while 2 out[f] stays below
 * reach - cutoff.  Waits for `stream`.
 * MDIR: the skin test of the drift (ExposeValidity.cpp;
 * docs/neighbor-groups.md, Section 7.1), here over a batch of frames. */
int32_t mdrtNbDisplacement(mdrtNb *ctx, const double *frames, int64_t count, const double box[3],
                           double *out, void *stream);

/* The same test in two halves, so that the caller can queue work between
 * them: mdrtNbDisplacementStart queues the test and the copy of its result
 * on `stream` without waiting; mdrtNbDisplacementResult waits for that copy
 * (not for the rest of the stream) and writes out[count] as
 * mdrtNbDisplacement.  A frames call queued in between reads the lists as
 * they are; the caller evaluates again, after a build, the frames that the
 * result puts past half the skin. */
int32_t mdrtNbDisplacementStart(mdrtNb *ctx, const double *frames, int64_t count, const double box[3],
                                void *stream);
int32_t mdrtNbDisplacementResult(mdrtNb *ctx, double *out);

/* Modes of mdrtNbParameterGradient. */
enum mdrtNbGradientMode {
  MDRT_NB_GRAD_PRODUCT = 0,  /* sum_k g_k . dF_k/dtheta for a cotangent g on the forces */
  MDRT_NB_GRAD_ENERGY = 1    /* dE/dtheta (pairs, excluded, reciprocal, self, background) */
};

/* The gradient of the term in its parameters at device positions x (f64
 * [n, 3]) with the lists of the last build (valid for x, box unchanged):
 * the charges of the atoms and the sigma / epsilon entries of the type-pair
 * table.  Adds dq_i to dq (device f64 [n], atom order) and d/dsigma_ab,
 * d/depsilon_ab to dtable (device f64 [2 ntypes^2]: the ntypes^2 sigma
 * entries, row-major by type pair, then the epsilon entries); both are
 * accumulated, so that frames add up.  MDRT_NB_GRAD_PRODUCT reads the
 * cotangent g (device f64 [n, 3], on the forces F = -dE/dx); for a loss
 * (1/K) sum |F - F_ref|^2, g = (2/K)(F - F_ref).  MDRT_NB_GRAD_ENERGY
 * ignores it and leaves out the dispersion correction, a host function of
 * the table.  The pair geometry is recomputed, not stored.  Refuses the
 * switched LJ form (MDRT_NB_UNSUPPORTED).  Asynchronous on `stream`.
 * MDIR: the force-matching product FrameEnergies.vjp(positions=)
 * (python/mdir/_frames.py:327, docs/python-frames.md:203-260, D381; its
 * cotangent is on dE/dx = -F) and the gradient in the tunables
 * (docs/python-gradient.md, D376), whose product refuses per-atom charges
 * with PME (D379); here they are given. */
int32_t mdrtNbParameterGradient(mdrtNb *ctx, const double *x, const double box[3],
                                const double *cotangent, int32_t mode, double *dq,
                                double *dtable, void *stream);

/* The force term of `count` frames, frame k at device positions
 * x + k x_stride (f64 [n, 3]) into forces + k f_stride, one after another
 * on `stream`, with the lists of the last build (valid for every frame):
 * the loop of mdrtNbForce calls of a frame evaluator in one call, since the
 * host's launch rate bounds a small frame's evaluation.  With `potentials`,
 * frame k's reciprocal potential grid goes to potentials + k p_stride (as
 * mdrtPmePotentialGrid).  MDRT_NB_ENERGY only with count 1 (the energies
 * are one evaluation's).  MDIR: FrameEvaluator's loop over the frames of a
 * call (python/mdir/_frames.py:769, D251).
 *
 * The launches of a call are kept as a CUDA graph (MDRT_NB_TUNE_FRAME_GRAPHS,
 * on by default) under a key of the call's arguments (pointers, strides,
 * count, cell, flags) and the state of the context (every buffer, capacity,
 * tuning value and build count): a call that repeats a key seen before is
 * one graph launch on `stream`.  A key is captured at its second call (the
 * first makes the lazy allocations outside any capture), and a context
 * keeps its 8 most recent keys.  The graph reads the inputs, the particle
 * tables and the lists at its launch, so new positions or parameters in the
 * same buffers need no new capture.  A call on a stream that is itself
 * being captured launches directly. */
int32_t mdrtNbForceFrames(mdrtNb *ctx, const double *x, int64_t x_stride, int64_t count, const double box[3],
                          uint32_t flags, double *forces, int64_t f_stride, float *potentials, int64_t p_stride,
                          void *stream);

/* mdrtNbParameterGradientPotential over `count` frames (positions
 * x + k x_stride, cotangents cotangent + k c_stride, potential grids
 * potentials + k p_stride or NULL), accumulating into dq and dtable.  In
 * the product mode the launches are kept as a graph, as those of
 * mdrtNbForceFrames. */
int32_t mdrtNbParameterGradientFrames(mdrtNb *ctx, const double *x, int64_t x_stride, int64_t count,
                                      const double box[3], const double *cotangent, int64_t c_stride, int32_t mode,
                                      const float *potentials, int64_t p_stride, double *dq, double *dtable,
                                      void *stream);

/* The reciprocal potential grid phi of the last force evaluation that ran
 * PME (K1 x K2 x K3 f32 in the grid's layout, the third index fastest) to
 * `grid` (device), asynchronous on `stream`; MDRT_NB_INVALID_ARGUMENT
 * without PME.  Kept for each frame, it spares the parameter gradient the
 * reciprocal forward (mdrtNbParameterGradientPotential).
 * MDIR: the potential grid of the PME stages (D231), which the vjp of
 * python/mdir/_frames.py:327 recomputes. */
int32_t mdrtPmePotentialGrid(mdrtNb *ctx, float *grid, void *stream);

/* mdrtNbParameterGradient with the potential grid phi that
 * mdrtPmePotentialGrid kept from the force evaluation at the same x,
 * charges and cell: the reciprocal forward is not run again.  phi NULL:
 * the same as mdrtNbParameterGradient.  A phi of other positions or
 * charges gives a wrong gradient; nothing checks it. */
int32_t mdrtNbParameterGradientPotential(mdrtNb *ctx, const double *x, const double box[3],
                                         const double *cotangent, int32_t mode, const float *phi,
                                         double *dq, double *dtable, void *stream);

/* A device pointer to a buffer of the neighbor structure and its element
 * count (a view; invalidated by the next build that grows).
 * MDIR: _mlir_ciface_mdrtGroupsBuffer(result, handle, slot),
 * runtime/mdrt_cuda.c:3109. */
int32_t mdrtNbGroupsBuffer(mdrtNb *ctx, int32_t slot, void **pointer, int64_t *count);

/* The graphs of the frames entries: captures and replays so far. */
int32_t mdrtNbFrameGraphInfo(mdrtNb *ctx, int64_t *captures, int64_t *replays);

/* The capacity C of a list (entries a group) and the builds / growths so far.
 * MDIR: mdrtGroupsBuilt, mdrt_cuda.c:3208. */
int32_t mdrtNbGroupsInfo(mdrtNb *ctx, int64_t *list_capacity, int64_t *builds, int64_t *grows);

/* The device status word (NB_STATUS_* bits: list overflow, fixed-point
 * overflow, non-finite positions, stale list, timeout); waits for stream.
 * clear != 0 resets it. */
int32_t mdrtNbStatus(mdrtNb *ctx, void *stream, int32_t clear, int32_t *status);

/* Average device time (ms, CUDA events on `stream`) of `iterations`
 * launches of each stage of the force term at device positions x, after a
 * valid build: out[0] frame gather, out[1] pair kernel, out[2] excluded
 * correction, out[3] PME (spread, FFTs, convolution, gather), out[4] force
 * finish, out[5] neighbor build (launches only), out[6] pruning (0 without
 * a dual list); out holds 8 doubles.  The launches of a stage are replayed
 * from a CUDA graph, so the host's launch rate does not enter the numbers.
 * For the roofline of each kernel; the forces it leaves are not meaningful.
 * MDIR: MDRT_WAIT=1 per-kernel timing (runtime/mdrt_cuda.c:600). */
int32_t mdrtNbTimeKernels(mdrtNb *ctx, const double *x, const double box[3], int32_t iterations,
                          void *stream, double *out);

/* ---- The MD step (leap-frog, SETTLE, Bussi thermostat) ------------------
 * MDIR: the compiled step loop that Simulation::run calls
 * (lib/Compiler/Simulation.cpp:421, 1679) and its replayed step graph
 * (runtime/mdrt_step_graph.cu), here for the nonbonded + PME system alone. */
typedef struct mdrtMd mdrtMd;

/* An integrator over the term `nb`: masses (host f64 [n], amu), and
 * `nwaters` rigid three-site waters (host int32 [nwaters][3]: O, H, H) held
 * by SETTLE at O-H d_oh and H-H d_hh (nm); the other atoms move freely. */
int32_t mdrtMdCreate(mdrtMd **out, mdrtNb *nb, const double *masses, int64_t nwaters,
                     const int32_t *waters, double d_oh, double d_hh);
int32_t mdrtMdDestroy(mdrtMd *md);
/* Bussi (CSVR) thermostat at `temperature` K with time constant tau (ps);
 * tau <= 0 leaves the energy constant (NVE).  `seed` fixes the noise.  The
 * velocity scaling a step computes for the next one is dropped: the next
 * step starts unscaled. */
int32_t mdrtMdSetThermostat(mdrtMd *md, double temperature, double tau, uint64_t seed);
/* The look-ahead of the rebuild decision: the drift's growth over the window
 * that ended is extrapolated `factor` times (default 1.5; 0: none).  A drift
 * past half the skin before the next decision stops the step (the steps
 * after it do nothing) and the host rebuilds there, so a smaller factor
 * costs stops, never a missed pair.  No MDIR counterpart: MDIR tests every
 * step on the device and rebuilds in its host loop (ExposeValidity.cpp). */
int32_t mdrtMdSetLookahead(mdrtMd *md, double factor);
/* A neighbor build at device positions x that also resets the reference
 * positions of the test of validity (D80). */
int32_t mdrtMdBuild(mdrtMd *md, const double *x, const double box[3], void *stream);
/* A new state x for mdrtMdRun (after the caller wrote new positions): when
 * every atom of x lies within half the skin of the positions of the last
 * build (the test that every step makes), the lists serve x; its frames are
 * made again, and the pruning that the step's update would ask for after
 * this drift is set (*built = 0).  Otherwise, or in another cell, a build
 * as mdrtMdBuild (*built = 1).  A state that the last run left, read back
 * and written again, keeps the lists, so that the run goes on as one
 * longer run would.  Waits for `stream`.  MDIR: the validity test of
 * ExposeValidity.cpp before its host loop rebuilds (D80). */
int32_t mdrtMdRefresh(mdrtMd *md, const double *x, const double box[3], void *stream, int32_t *built);
/* `steps` leap-frog steps of dt (ps) on the device state x, v (f64 [n, 3]).
 * The lists are pruned on the device whenever 2 max|x - x_prune| > R_in - r_c
 * (gated launches in every step) and rebuilt at the end of each window of
 * steps (`unroll` steps in a graph, 10 step by step) when the drift could
 * pass half the skin before the next decision: 2 (d + factor (d - d_last)
 * + 0.002 nm) > R - r_c, d = max|x - x_build| (mdrtMdSetLookahead).  A drift
 * past half the skin inside a window stops the step there (the later steps
 * of the graphs do nothing); the host rebuilds at that step and runs the
 * steps left.  unroll > 0 replays a CUDA graph of `unroll` steps
 * (one conditional node, the rebuild; no host wait inside); unroll < 0 runs
 * step by step with a decision every -unroll steps (10 for unroll = 0); the
 * steps after the last whole graph run step by step with the graph's window;
 * the run of graphs
 * starts from a checkpoint of x, v and the thermostat state and ends in one
 * host wait that reads what its rebuilds saw: after a list that outgrew its
 * capacity the run is redone from the checkpoint with grown lists
 * (count-then-grow, MDIR MDExecToGPU.cpp:10107-10175), and positions that
 * are not finite return MDRT_NB_NAN_POSITION.  unroll = 0 runs step by step,
 * the host reading the test of validity after each step. */
int32_t mdrtMdRun(mdrtMd *md, double *x, double *v, const double box[3], double dt, int64_t steps,
                  int32_t unroll, void *stream);
/* The integrator of mdrtMdRun: leap-frog (the default; v half a step
 * behind x) or velocity Verlet (v on the step at the start and the end of
 * each run; the same positions).  Velocity Verlet refuses rigid waters
 * (MDRT_NB_UNSUPPORTED): velocities on the step would need their velocity
 * constraints.  MDIR: the integrators of docs/dynamics.md (velocity Verlet
 * for argon.test; leap-frog). */
enum mdrtMdIntegrator { MDRT_MD_LEAP_FROG = 0, MDRT_MD_VELOCITY_VERLET = 1 };
int32_t mdrtMdSetIntegrator(mdrtMd *md, int32_t method);
/* out[9]: thermostat scaling, kinetic energy of the last two half steps,
 * steps taken, builds made, degrees of freedom, prunings made, runs of step
 * graphs redone after a list overflow, stops at a drift past half the skin
 * between two rebuild decisions; waits for `stream`. */
int32_t mdrtMdThermo(mdrtMd *md, void *stream, double *out);
/* The device array of the forces of the last step (f64 [n, 3]). */
int32_t mdrtMdForces(mdrtMd *md, double **forces);

/* ---- An entry point that allocates nothing -------------------------------
 * mdrtNbExcludedNoAlloc: the excluded-pair Ewald correction
 * -f q_i q_j erf(beta r)/r over `npairs` pairs (device int32 [npairs][2],
 * i < j), in f64 from device positions x (f64 [n, 3]) and charges (f64 [n]),
 * in the orthorhombic cell box[3] (host).  Adds the forces to `forces`
 * (device f64 [n, 3]) and writes the energy and the virial (xx yy zz xy xz
 * yz) to energy_virial (device f64 [7]); asynchronous on `stream`.
 *
 * For callers that cannot allocate device memory: host programs (and
 * plugins inside them) that own all device memory through a fixed pool and
 * forbid other allocations, and loops that must not pay the device
 * synchronization of cudaFree.  It calls no cudaMalloc, cudaFree or
 * allocating library routine: its scratch (the per-block partial sums) is a
 * fixed __device__ array of the library, held on every GPU that loads it
 * until the process exits.  More than MDRT_NB_NOALLOC_MAX_PAIRS pairs is
 * refused with MDRT_NB_INVALID_ARGUMENT (and a message on stderr).  The
 * first call on a device looks up the array's device address (a runtime
 * query, no allocation) and keeps it for the life of the process; make that
 * first call before any stream capture, and do not call the entry point on
 * a device after a cudaDeviceReset of it (the kept address may be stale).
 * Calls share the array: two calls that overlap on the GPU race.
 * No counterpart in MDIR; the allocating path is mdrtNbForce with
 * MDRT_NB_NO_PAIRS | MDRT_NB_NO_PME. */
#define MDRT_NB_NOALLOC_MAX_PAIRS (1 << 20)
int32_t mdrtNbExcludedNoAlloc(const double *x, const double *charges, const int32_t *pairs, int64_t npairs,
                              const double box[3], double beta, double coulomb, double *forces,
                              double *energy_virial, void *stream);

/* 3D real FFTs of a grid in f32 on `stream`, plans cached per size.
 * MDIR: _mlir_ciface_mdrtCudaFFTForward3DF32 / Backward3DF32
 * (runtime/mdrt_cuda.c:2942-2979), with plain pointers.  The backward
 * transform is not normalized and overwrites the half-complex grid. */
int32_t mdrtCudaFFTForward3DF32(const float *real, float *complex_out, int64_t k1, int64_t k2,
                                int64_t k3, void *stream);
int32_t mdrtCudaFFTBackward3DF32(float *complex_in, float *real_out, int64_t k1, int64_t k2,
                                 int64_t k3, void *stream);

/* ---- Batches of frames (the batching form) --------------------------------
 * Many independent systems ("frames") of uneven sizes, each with its own
 * orthorhombic cell and PME grid, evaluated together: the atoms of frame f
 * are atoms atom0[f] .. atom0[f+1]-1 of the batch (frames one after the
 * other), and every stage (the build, the pair kernel, the excluded pairs,
 * PME) is one launch over all frames, the pair kernel one persistent grid
 * over the units of every frame.  The frames share the interaction (cutoff,
 * reach, beta), the LJ type table and the spline order.  Deterministic mode,
 * the dual list and the switched LJ form are not offered for batches.
 * MDIR: frames are evaluated one after another (D251,
 * docs/python-frames.md:1178), its device batch (D386, docs/driver.md:
 * 1655-1700; python/mdir/_frames.py:769) loops over frames of one program. */
typedef struct mdrtNbBatch mdrtNbBatch;

/* A batch of `frames` frames with atoms[f] atoms each (host). */
int32_t mdrtNbBatchCreate(mdrtNbBatch **out, int32_t device, int32_t frames, const int64_t *atoms);
int32_t mdrtNbBatchDestroy(mdrtNbBatch *batch);
/* As mdrtNbSetParticles over all atoms of the batch; one type table. */
int32_t mdrtNbBatchSetParticles(mdrtNbBatch *batch, const double *charges, const int32_t *types,
                                int32_t ntypes, const double *sigma, const double *epsilon);
/* As mdrtNbSetExclusions in the batch's numbering; every pair inside one
 * frame (else MDRT_NB_INVALID_ARGUMENT). */
int32_t mdrtNbBatchSetExclusions(mdrtNbBatch *batch, const int32_t *offsets, const int32_t *partners);
int32_t mdrtNbBatchSetInteraction(mdrtNbBatch *batch, double cutoff, double reach, double beta,
                                  double coulomb);
/* The PME grid of each frame, grids[3 f + k] (host), and the spline order
 * (4 or 8).  Frames of one shape share one batched cuFFT plan pair. */
int32_t mdrtNbBatchPmeSetup(mdrtNbBatch *batch, const int32_t *grids, int32_t order);
/* MDRT_NB_TUNE_PAIR_BLOCKS_PER_SM (1-4) and MDRT_NB_TUNE_SEARCH_WARPS (1 or
 * 4 warps a group in the search); results do not depend on them. */
int32_t mdrtNbBatchSetTuning(mdrtNbBatch *batch, int32_t key, int32_t value);
/* The build of all frames at device positions x (f64 [n, 3], the batch's
 * numbering) in the cells boxes[3 f + k] (host); grows and builds again
 * until every list fits (host wait), as mdrtNbBuild. */
int32_t mdrtNbBatchBuild(mdrtNbBatch *batch, const double *x, const double *boxes, void *stream,
                         int32_t *sizes_out);
/* Forces of all frames (device f64 [n, 3]); flags as mdrtNbForce, plus
 * MDRT_NB_GRAPH: the launches captured once as a CUDA graph and replayed
 * (captured again when the buffers, pointers or flags change).  With
 * MDRT_NB_ENERGY the energies of each frame are summed in a fixed order. */
int32_t mdrtNbBatchForce(mdrtNbBatch *batch, const double *x, uint32_t flags, double *forces, void *stream);
/* out[f * MDRT_NB_E_COUNT + slot]: the energies and virials of each frame
 * (slots of mdrtNbEnergySlot) of the last MDRT_NB_ENERGY evaluation; waits. */
int32_t mdrtNbBatchEnergies(mdrtNbBatch *batch, void *stream, double *out);
/* out[2 f]: the Ewald self term of frame f, out[2 f + 1] its background
 * term (host, f64), in the cells of the last build. */
int32_t mdrtNbBatchConstants(mdrtNbBatch *batch, double *out);
/* The project's autotuner: times a build and an evaluation with energies
 * for every search width (4, 1 warps a group), pair-kernel occupancy (4..1
 * blocks per SM) and staging depth (1, 2), keeps the fastest, and writes it
 * to choice[3] = {search warps, pair blocks per SM, staging depth}.  The
 * members of a group (16, the column places of the build) and the threads
 * an i-cluster's accumulators rotate over (16, a half-warp) are fixed by
 * the layout.  Needs a build (for the cells);
 * `forces` is scratch (device f64 [n, 3]).  No MDIR counterpart: MDIR's
 * launch shapes are fixed by its emitters (DevicePolicy.cpp:72-99). */
int32_t mdrtNbBatchAutotune(mdrtNbBatch *batch, const double *x, double *forces, void *stream,
                            int32_t *choice);

/* ---- MDIR's own runtime names ----------------------------------------------
 * The entries an MDIR host program binds for the groups and the cuFFT
 * transforms, with the memref descriptors of MLIR's C interface (a buffer
 * of rank 1 or 2: allocated and aligned pointers, offset, sizes, strides;
 * runtime/mdrt_cuda.c:1530-1582).  Where MDIR aborts (an invalid slot, a
 * failed allocation, a failed transform), these entries print to stderr,
 * leave an empty descriptor, and keep the status for mdrtGroupsLastStatus. */
typedef struct {
  void *allocated;
  void *aligned;
  int64_t offset;
  int64_t size;
  int64_t stride;
} mdrtMemRef1D;
typedef struct {
  void *allocated;
  void *aligned;
  int64_t offset;
  int64_t sizes[2];
  int64_t strides[2];
} mdrtMemRef2D;

/* The slots of a groups registry, MDIR's stable slot table (ABI version 3,
 * include/mdir/Runtime/GroupsABI.h:10-44); every slot a buffer of 32-bit
 * values whose length follows from the registry's places and blocks. */
#define MDRT_GROUPS_ABI_VERSION 3
enum mdrtGroupsSlot {
  MDRT_GROUPS_ORDER = 0,          /* [places] the particle at each place, -1 empty */
  MDRT_GROUPS_COUNTS = 1,         /* [places / 16] entries of each group's list */
  MDRT_GROUPS_ENTRIES = 2,        /* [64 blocks] the partner place of each entry, -1 past a list's end */
  MDRT_GROUPS_MASKS = 3,          /* [64 blocks] members (bits 0-15) | image (bits 16-30, this header's code) */
  MDRT_GROUPS_UNIT_GROUPS = 4,    /* [blocks] the group of each block */
  MDRT_GROUPS_UNIT_ORDINALS = 5,  /* [blocks] the block's number in its group's list */
  MDRT_GROUPS_SHIFTS = 6,         /* [places] whole cells of each place, int8x4 */
  MDRT_GROUPS_INNER_ENTRIES = 7,  /* [64 blocks] the pruned lists by blocks */
  MDRT_GROUPS_INNER_MASKS = 8,
  MDRT_GROUPS_INNER_COUNTS = 9,   /* [blocks] entries of each block of the pruned lists */
  MDRT_GROUPS_BLOCK_OF = 10,      /* [mdrtGroupsReserveBlockOf's length] */
  MDRT_GROUPS_ACTIVE_UNITS = 11,  /* [blocks] the blocks of the pruned lists that hold entries */
  MDRT_GROUPS_ACTIVE_COUNT = 12,  /* [1] their number */
  MDRT_GROUPS_ACTIVE_RUNS = 13,
  MDRT_GROUPS_ACTIVE_WIDE_RUNS = 14,
  MDRT_GROUPS_PLACED = 15,        /* [places, 3] f32 positions of the places in the frames of the build */
  MDRT_GROUPS_SEGMENT_COUNTS = 16,
  MDRT_GROUPS_SEGMENT_LAST = 17,
  MDRT_GROUPS_SEGMENT_ORDER = 18,
  MDRT_GROUPS_RECORD_ENTRIES = 19,
  MDRT_GROUPS_RECORD_MASKS = 20,
  MDRT_GROUPS_RECORD_GROUPS = 21,
  MDRT_GROUPS_RECORD_COUNTS = 22,
  MDRT_GROUPS_SEGMENT_OFFSETS = 23,
  MDRT_GROUPS_BUFFERS = 24
};

/* A registry with room for `places` places (rounded up to 16) and `blocks`
 * blocks of 64 entries on the current device; the outer list's slots (0-6)
 * are allocated now, the others where first asked for.  Returns the handle,
 * 0 on failure.  MDIR: mdrtGroupsCreate, runtime/mdrt_cuda.c:3087. */
int64_t mdrtGroupsCreate(int64_t places, int64_t blocks);
/* The buffer of `slot` as a memref of rank 1 (allocated at its first use).
 * MDIR: _mlir_ciface_mdrtGroupsBuffer, mdrt_cuda.c:3109. */
void _mlir_ciface_mdrtGroupsBuffer(mdrtMemRef1D *result, int64_t handle, int64_t slot);
/* Room for `places` places and `blocks` blocks, a quarter more than asked,
 * if the registry has less; what the buffers held is lost (waits for the
 * device).  MDIR: mdrtGroupsGrow, mdrt_cuda.c:3185. */
void mdrtGroupsGrow(int64_t handle, int64_t places, int64_t blocks);
/* After a complete build: the growths of the lists since the last call,
 * and the registry marked built.  MDIR: mdrtGroupsBuilt, mdrt_cuda.c:3208. */
int64_t mdrtGroupsBuilt(int64_t handle);
/* Room for `length` values of MDRT_GROUPS_BLOCK_OF, a quarter more than
 * asked, if it has less.  MDIR: mdrtGroupsReserveBlockOf, mdrt_cuda.c:3218. */
void mdrtGroupsReserveBlockOf(int64_t handle, int64_t length);
/* The placed positions as a memref of rank 2, [places, 3] f32.
 * MDIR: _mlir_ciface_mdrtGroupsPlaced, mdrt_cuda.c:3300. */
void _mlir_ciface_mdrtGroupsPlaced(mdrtMemRef2D *result, int64_t handle);
/* Frees a registry (MDIR releases them when its run ends).  No MDIR
 * counterpart by name. */
int32_t mdrtGroupsDestroy(int64_t handle);
/* The status the last failing MDIR-named entry left (MDRT_NB_OK if none
 * since the last call), then cleared.  No MDIR counterpart: MDIR aborts. */
int32_t mdrtGroupsLastStatus(void);
/* Copies the lists of the context's last build into the registry's slots
 * in MDIR's layout (growing it first as mdrtGroupsGrow does): order,
 * counts, entries and masks in blocks of 64 with each block's group and
 * ordinal, shifts, the placed positions, and, after a pruning, the pruned
 * lists by blocks with the entries each holds, the active blocks (all of
 * them) and their number.  Asynchronous on `stream` (one host wait for the
 * count of the pruned blocks).  The values are this library's (partner
 * places, 16-member masks with this header's image code, centred frames).
 * No MDIR counterpart by name: MDIR's emitted build writes the registry. */
int32_t mdrtNbGroupsExport(mdrtNb *ctx, int64_t handle, void *stream);
/* The stream of the MDIR-named transforms below, which take none (NULL:
 * the default stream). */
int32_t mdrtNbSetAbiStream(void *stream);
/* The forward and the backward (not normalized) 3D real transforms in f32
 * of a k1 x k2 x k3 grid and its k1 x k2 x (k3/2 + 1) half-complex grid.
 * MDIR: _mlir_ciface_mdrtCudaFFTForward3DF32 / Backward3DF32,
 * runtime/mdrt_cuda.c:2942-2979. */
void _mlir_ciface_mdrtCudaFFTForward3DF32(mdrtMemRef1D *real, mdrtMemRef1D *complex, int64_t k1, int64_t k2,
                                          int64_t k3);
void _mlir_ciface_mdrtCudaFFTBackward3DF32(mdrtMemRef1D *complex, mdrtMemRef1D *real, int64_t k1, int64_t k2,
                                           int64_t k3);
/* The backward transform of the half-complex grid times the Gaussian
 * influence of a rectangular cell given by per-axis tables: for axis a of
 * k_a points, three rows of k_a f32 (its wave numbers, their squares m_a^2
 * and its factors t_a), the axes one after the other; each point (x, y, z)
 * is scaled by t_1[x] t_2[y] t_3[z] / (m_1^2[x] + m_2^2[y] + m_3^2[z]) (0
 * where the squares sum to 0), then transformed back.  MDIR:
 * _mlir_ciface_mdrtCudaFFTGaussianBackwardF32 (mdrt_cuda.c:2985-2990) with
 * its load callback (runtime/pme_callback.cu:5-21). */
void _mlir_ciface_mdrtCudaFFTGaussianBackwardF32(mdrtMemRef1D *complex, mdrtMemRef1D *real, mdrtMemRef1D *tables,
                                                 int64_t k1, int64_t k2, int64_t k3);

#ifdef __cplusplus
}
#endif

#endif /* MDRT_NB_H */
