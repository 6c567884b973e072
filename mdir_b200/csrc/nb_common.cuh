// Shared definitions of the sm_100a short-range nonbonded + PME library.
//
// Layout in HBM (one context = one system on one device):
//   places     P = 16 * groups; place p holds atom order[p] or -1 (empty).
//              A group is 16 consecutive places of one column of the grid,
//              sorted along z (the spatial cell sort of the build).
//   frames     xq[p] = float4(x + (S_p - 1/2) L rounded once to f32, q);
//              S_p is the whole-cell shift that took the atom into the cell
//              at the last build (kept per place, three int8 in shift_p).
//              The frames are centred on the cell: the largest coordinate,
//              and so the spacing of f32 values, is half that of [0, L);
//              pair displacements do not depend on the origin, and readers
//              of absolute positions (PME) add the half cell back.
//   lists      one slab of C entries per group: entry = int2(q, bits) with
//              q the partner place, bits 0-15 the members that pair with it
//              and bits 16-30 the lattice vector of the partner's image, 5
//              bits a component (NB_IMAGE_BITS below).  A pruned (inner)
//              list holds its entries in classes: those with more than
//              NB_SPARSE_BITS members first, then those with 1, 2, ...,
//              NB_SPARSE_BITS members (a list too long for the pruning's
//              shared-memory staging keeps the outer order; the pair kernel
//              is right in either order).
//   units      (group, ordinal) work items of 64 entries each, in group
//              order, so that every launch sees them in the same order.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define NB_GROUP 16
#define NB_UNIT 64
#define NB_WARP 32
// Entries with at most this many members are evaluated member by member
// (a round of 32 such entries takes as many steps as its largest entry has
// members) instead of in the 16 rotating steps of a dense round.
#define NB_SPARSE_BITS 5

// sizes[] slots written by the build (device) and read by the host.
enum NbSizeSlot {
  NB_SIZE_PLACES = 0,     // places the build needed (16 * groups)
  NB_SIZE_LONGEST = 1,    // longest list of a group (entries)
  NB_SIZE_UNITS = 2,      // units of 64 entries
  NB_SIZE_EXCL_WIDE = 3,  // groups whose excluded partners did not fit smem
  NB_SIZE_NAN = 4,        // positions that are not finite or far outside
  NB_SIZE_OVERFLOW = 5,   // 1 if any buffer was too small (nothing past it written)
  NB_SIZE_GROUPS = 6,     // groups used
  NB_SIZE_ENTRIES = 7,    // total entries written
  NB_SIZE_COUNT = 8
};

// Device status word bits (mdrtNbStatus).
enum NbStatusBits {
  NB_STATUS_LIST_OVERFLOW = 1,
  NB_STATUS_FIXED_OVERFLOW = 2,
  NB_STATUS_NAN = 4,
  NB_STATUS_STALE_LIST = 8,
  NB_STATUS_TIMEOUT = 16,
};

struct NbBox {
  float L[3];      // edges in f32
  double Ld[3];    // edges in f64
};

// The multiple of the cell edge added to an atom's position in its frame:
// its whole-cell shift less the half cell of the centred frames.
__host__ __device__ inline double nb_frame_shift(int s) { return (double)s - 0.5; }

// The image of an entry: a lattice vector n = (na, nb, nc) of the cell,
// each component + 16 in five bits (bits 16-30 of the entry's second word;
// -16..15, since a triclinic brick spans up to 3.5 periods of a).
#define NB_IMAGE_BITS 0x7fff
__host__ __device__ inline int nb_image_code(int sx, int sy, int sz) {
  return (sx + 16) | ((sy + 16) << 5) | ((sz + 16) << 10);
}

__device__ __forceinline__ void nb_decode_image(int code, int &sx, int &sy, int &sz) {
  sx = (code & 31) - 16;
  sy = ((code >> 5) & 31) - 16;
  sz = ((code >> 10) & 31) - 16;
}

// The cell: rows a = (ax, 0, 0), b = (bx, by, 0), c = (cx, cy, cz) of a
// lower-triangular H (an orthorhombic cell has no tilts bx, cx, cy).
struct NbCell {
  float ax, by, cz, bx, cx, cy;
};

// The lattice vector n H in f32, each product and each sum rounded in this
// order: ((na ax + nb bx) + nc cx, nb by + nc cy, nc cz).  The neighbor
// test of the build shifts by exactly this (its pair sets are compared bit
// for bit); without tilts it is (na ax, nb by, nc cz).
__device__ __forceinline__ float3 nb_lattice_shift(int na, int nb, int nc, const NbCell &H) {
  float fa = (float)na, fb = (float)nb, fc = (float)nc;
  float tx = __fadd_rn(__fadd_rn(__fmul_rn(fa, H.ax), __fmul_rn(fb, H.bx)), __fmul_rn(fc, H.cx));
  float ty = __fadd_rn(__fmul_rn(fb, H.by), __fmul_rn(fc, H.cy));
  float tz = __fmul_rn(fc, H.cz);
  return make_float3(tx, ty, tz);
}

// Fixed-point scale of the deterministic force accumulators: 2^32 units
// per kJ/mol/nm.
#define NB_FORCE_SCALE 4294967296.0
#define NB_FORCE_SCALE_INV (1.0 / 4294967296.0)
// Fixed-point scale of the deterministic PME grid: 2^40 per e.
#define NB_GRID_SCALE 1099511627776.0

// Programmatic dependent launch (sm_90 and newer): a kernel launched with
// nb_launch_chained may start while the kernel before it on its stream is
// finishing; it calls nb_grid_wait() before it reads anything that kernel
// (or one before it) writes, and every such kernel waits in at least one
// thread, so that its completion still implies theirs.  The wait is a no-op
// for a kernel launched the ordinary way.  In a captured graph the launch
// becomes a programmatic edge, which hides most of the launch gap between
// the dependent kernels of the MD step.
__device__ __forceinline__ void nb_grid_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
// Lets the chained kernel after this one launch once every block of this
// grid has called it (or exited): the dependent's blocks then run their work
// before nb_grid_wait() beside this kernel's.  Called by a persistent kernel
// whose blocks are all resident, it cannot hold back blocks of its own grid.
__device__ __forceinline__ void nb_grid_launch_dependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... KArgs, typename... Args>
static inline cudaError_t nb_launch_chained(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                                            cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}
