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
#include <cmath>
#include <cstdio>
#include <vector>

#include "../../include/mdrt_nb.h"
#include "nb_context.h"

struct mdrtMd {
  NbCtx *nb = nullptr;
  mdrtNb *handle = nullptr;
  int64_t n = 0, nwaters = 0, nfree = 0;
  double *inv_mass = nullptr;      // device f64 [n]
  double *mass = nullptr;          // device f64 [n]
  int32_t *waters = nullptr;       // device [nw][3] (O, H1, H2)
  int32_t *free_atoms = nullptr;   // device [nfree]
  double dOH = 0.09572, dHH = 0.15139, mO = 15.9994, mH = 1.008;
  double *force = nullptr;         // device f64 [n, 3]
  double *x_ref = nullptr;         // positions at the last build
  double *ke_part = nullptr;       // per-block kinetic partials
  int ke_blocks = 0;
  unsigned int *maxd2 = nullptr;   // float bits of max |x - x_ref|^2
  double *thermo = nullptr;        // [0] lambda, [1] KE of the last half step, [2] KE before, [3] steps, [4] builds
  double temperature = 300.0, tau = 0.0;
  int64_t ndof = 0;
  unsigned long long seed = 1;
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
__device__ __forceinline__ Vec3 v3(double x, double y, double z) { return {x, y, z}; }
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

// SETTLE: the constrained positions a3, b3, c3 of one water from its
// constrained old positions a0, b0, c0 and unconstrained new a1, b1, c1.
__device__ void settle(const SettleParams &P, Vec3 a0, Vec3 b0, Vec3 c0, Vec3 &a1, Vec3 &b1, Vec3 &c1) {
  double M = P.mO + 2.0 * P.mH;
  Vec3 d = (1.0 / M) * (P.mO * a1 + P.mH * b1 + P.mH * c1);  // centre of mass of the new positions
  Vec3 A1 = a1 - d, B1 = b1 - d, C1 = c1 - d;
  Vec3 B0 = b0 - a0, C0 = c0 - a0;
  Vec3 ez = unit(cross(B0, C0));      // normal of the old plane
  Vec3 ex = unit(cross(A1, ez));      // perpendicular to it and to the new O
  Vec3 ey = cross(ez, ex);
  // the old and new sites in the frame (ex, ey, ez)
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

__device__ __forceinline__ void atomic_max_float(unsigned int *addr, float v) {
  atomicMax(addr, __float_as_uint(fmaxf(v, 0.f)));  // non-negative floats order as integers
}

// One leap-frog step with SETTLE: v += lambda-scaled, f/m dt; x += v dt;
// constrain; v = (x_new - x_old)/dt.  A thread per water, then per free atom.
__global__ void md_update(int64_t nwaters, int64_t nfree, const int32_t *__restrict__ waters,
                          const int32_t *__restrict__ free_atoms, SettleParams S,
                          const double *__restrict__ inv_mass, const double *__restrict__ mass,
                          const double *__restrict__ f, double *__restrict__ x, double *__restrict__ v,
                          const double *__restrict__ x_ref, const double *__restrict__ thermo, double dt,
                          double *__restrict__ ke_part, unsigned int *__restrict__ maxd2) {
  __shared__ double s_ke[8];
  __shared__ float s_d2[8];
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double lambda = thermo[0];
  double ke = 0.0;
  float d2max = 0.f;
  if (t < nwaters) {
    int ia = waters[3 * t], ib = waters[3 * t + 1], ic = waters[3 * t + 2];
    Vec3 a0 = load3(x, ia), b0 = load3(x, ib), c0 = load3(x, ic);
    Vec3 va = lambda * load3(v, ia) + (dt * inv_mass[ia]) * load3(f, ia);
    Vec3 vb = lambda * load3(v, ib) + (dt * inv_mass[ib]) * load3(f, ib);
    Vec3 vc = lambda * load3(v, ic) + (dt * inv_mass[ic]) * load3(f, ic);
    Vec3 a1 = a0 + dt * va, b1 = b0 + dt * vb, c1 = c0 + dt * vc;
    settle(S, a0, b0, c0, a1, b1, c1);
    double inv_dt = 1.0 / dt;
    va = inv_dt * (a1 - a0);
    vb = inv_dt * (b1 - b0);
    vc = inv_dt * (c1 - c0);
    store3(x, ia, a1);
    store3(x, ib, b1);
    store3(x, ic, c1);
    store3(v, ia, va);
    store3(v, ib, vb);
    store3(v, ic, vc);
    ke = 0.5 * (mass[ia] * dot(va, va) + mass[ib] * dot(vb, vb) + mass[ic] * dot(vc, vc));
    Vec3 da = a1 - load3(x_ref, ia), db = b1 - load3(x_ref, ib), dc = c1 - load3(x_ref, ic);
    d2max = (float)fmax(dot(da, da), fmax(dot(db, db), dot(dc, dc)));
  } else if (t < nwaters + nfree) {
    int i = free_atoms[t - nwaters];
    Vec3 vi = lambda * load3(v, i) + (dt * inv_mass[i]) * load3(f, i);
    Vec3 xi = load3(x, i) + dt * vi;
    store3(x, i, xi);
    store3(v, i, vi);
    ke = 0.5 * mass[i] * dot(vi, vi);
    Vec3 di = xi - load3(x_ref, i);
    d2max = (float)dot(di, di);
  }
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ke += __shfl_xor_sync(0xffffffffu, ke, o);
    d2max = fmaxf(d2max, __shfl_xor_sync(0xffffffffu, d2max, o));
  }
  if (lane == 0) {
    s_ke[warp] = ke;
    s_d2[warp] = d2max;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    float m = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      s += s_ke[w];
      m = fmaxf(m, s_d2[w]);
    }
    ke_part[blockIdx.x] = s;
    atomic_max_float(maxd2, m);
  }
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
  return sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2);
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

// The kinetic energy of the half step (fixed-order sum) and the Bussi
// (CSVR; Bussi, Donadio & Parrinello, J. Chem. Phys. 126 (2007) 014101)
// scaling for the next update.  thermo: [0] lambda, [1] KE, [2] KE before,
// [3] steps, [4] builds.
__global__ void md_thermostat(const double *__restrict__ ke_part, int nblocks, double *thermo, double dt,
                              double tau, double temperature, double ndof, unsigned long long seed) {
  __shared__ double s[256];
  double v = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) v += ke_part[b];
  s[threadIdx.x] = v;
  __syncthreads();
  for (int stride = blockDim.x / 2; stride > 0; stride >>= 1) {
    if ((int)threadIdx.x < stride) s[threadIdx.x] += s[threadIdx.x + stride];
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  double K = s[0];
  thermo[2] = thermo[1];
  thermo[1] = K;
  double step = thermo[3];
  thermo[3] = step + 1.0;
  double lambda = 1.0;
  if (tau > 0.0 && K > 0.0 && ndof > 1.0) {
    const double kB = 0.0083144626181532;
    double Kt = 0.5 * ndof * kB * temperature;
    double c = exp(-dt / tau);
    unsigned long long ctr = (unsigned long long)step * 1024ull;
    double r1 = normal01(ctr, seed);
    double sum = 2.0 * gamma_draw(0.5 * (ndof - 1.0), ctr, seed);
    double Knew = K + (1.0 - c) * (Kt * (r1 * r1 + sum) / ndof - K) + 2.0 * r1 * sqrt(c * (1.0 - c) * K * Kt / ndof);
    lambda = sqrt(fmax(Knew, 0.0) / K);
  }
  thermo[0] = lambda;
}

// Sets the conditional of the rebuild: 2 max|x - x_ref| > R - r_c (D80, in
// a cell that does not change).
__global__ void md_check(unsigned int *maxd2, double half_skin2, cudaGraphConditionalHandle h, int use_graph,
                         int *flag) {
  float d2 = __uint_as_float(*maxd2);
  int rebuild = (double)d2 > half_skin2 ? 1 : 0;
  if (flag) *flag = rebuild;
  if (use_graph) cudaGraphSetConditional(h, rebuild);
}

// After a build: the reference positions and the counters.
__global__ void md_after_build(int64_t n3, const double *__restrict__ x, double *__restrict__ x_ref,
                               unsigned int *maxd2, double *thermo, const int32_t *sizes, int *status) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n3) x_ref[k] = x[k];
  if (k == 0) {
    *maxd2 = 0u;
    thermo[4] += 1.0;
    if (sizes[NB_SIZE_OVERFLOW] != 0) atomicOr(status, NB_STATUS_LIST_OVERFLOW);
    if (sizes[NB_SIZE_NAN] != 0) atomicOr(status, NB_STATUS_NAN);
  }
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

// One step on `s`: forces at x, update, thermostat, the test of validity;
// with a graph the rebuild is a conditional node added by the caller.
static void md_step_body(mdrtMd &m, double *x, double *v, const double box[3], double dt, cudaStream_t s,
                         cudaGraphConditionalHandle h, int use_graph, int *flag) {
  NbCtx &c = *m.nb;
  nb_gather_frames(c, x, box, s);
  nb_pairs_run(c, box, false, s);
  nb_excluded_run(c, box, false, s);
  if (c.pme.on && c.beta > 0.0) nb_pme_run(c, box, false, false, s);
  nb_finish_forces(c, m.force, 0, s);
  int64_t units = m.nwaters + m.nfree;
  cudaMemsetAsync(m.maxd2, 0, sizeof(unsigned int), s);
  md_update<<<m.ke_blocks, 256, 0, s>>>(m.nwaters, m.nfree, m.waters, m.free_atoms, settle_params(m),
                                       m.inv_mass, m.mass, m.force, x, v, m.x_ref, m.thermo, dt, m.ke_part,
                                       m.maxd2);
  (void)units;
  md_thermostat<<<1, 256, 0, s>>>(m.ke_part, m.ke_blocks, m.thermo, dt, m.tau, m.temperature, (double)m.ndof,
                                  m.seed);
  double half = 0.5 * (c.reach - c.cutoff);
  md_check<<<1, 1, 0, s>>>(m.maxd2, half * half, h, use_graph, flag);
}

static void md_rebuild_body(mdrtMd &m, const double *x, const double box[3], cudaStream_t s) {
  NbCtx &c = *m.nb;
  nb_build_launch_public(c, x, box, s);
  md_after_build<<<blocks_for(3 * m.n, 256), 256, 0, s>>>(3 * m.n, x, m.x_ref, m.maxd2, m.thermo, c.sizes,
                                                         c.status);
}

static void md_free(mdrtMd *m) {
  if (!m) return;
  if (m->exec) cudaGraphExecDestroy(m->exec);
  if (m->graph) cudaGraphDestroy(m->graph);
  for (void *p : {(void *)m->inv_mass, (void *)m->mass, (void *)m->waters, (void *)m->free_atoms,
                  (void *)m->force, (void *)m->x_ref, (void *)m->ke_part, (void *)m->maxd2, (void *)m->thermo})
    if (p) cudaFree(p);
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
  m->n = c.n;
  m->nwaters = nwaters;
  m->dOH = d_oh;
  m->dHH = d_hh;
  std::vector<char> in_water(c.n, 0);
  for (int64_t w = 0; w < nwaters; ++w)
    for (int k = 0; k < 3; ++k) {
      int32_t a = waters[3 * w + k];
      if (a < 0 || a >= c.n || in_water[a]) {
        md_free(m);
        return MDRT_NB_INVALID_ARGUMENT;
      }
      in_water[a] = 1;
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
  std::vector<int32_t> fr;
  for (int64_t i = 0; i < c.n; ++i)
    if (!in_water[i]) fr.push_back((int32_t)i);
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
  m->ke_blocks = blocks_for(nwaters + m->nfree, 256);
  bool ok = cudaMalloc(&m->inv_mass, sizeof(double) * c.n) == cudaSuccess &&
            cudaMalloc(&m->mass, sizeof(double) * c.n) == cudaSuccess &&
            cudaMalloc(&m->waters, sizeof(int32_t) * std::max<int64_t>(3 * nwaters, 1)) == cudaSuccess &&
            cudaMalloc(&m->free_atoms, sizeof(int32_t) * std::max<int64_t>(m->nfree, 1)) == cudaSuccess &&
            cudaMalloc(&m->force, sizeof(double) * 3 * c.n) == cudaSuccess &&
            cudaMalloc(&m->x_ref, sizeof(double) * 3 * c.n) == cudaSuccess &&
            cudaMalloc(&m->ke_part, sizeof(double) * m->ke_blocks) == cudaSuccess &&
            cudaMalloc(&m->maxd2, sizeof(unsigned int)) == cudaSuccess &&
            cudaMalloc(&m->thermo, sizeof(double) * 8) == cudaSuccess;
  if (!ok) {
    md_free(m);
    return MDRT_NB_CUDA_ERROR;
  }
  cudaMemcpy(m->inv_mass, inv.data(), sizeof(double) * c.n, cudaMemcpyHostToDevice);
  cudaMemcpy(m->mass, masses, sizeof(double) * c.n, cudaMemcpyHostToDevice);
  if (nwaters > 0) cudaMemcpy(m->waters, waters, sizeof(int32_t) * 3 * nwaters, cudaMemcpyHostToDevice);
  if (m->nfree > 0) cudaMemcpy(m->free_atoms, fr.data(), sizeof(int32_t) * m->nfree, cudaMemcpyHostToDevice);
  double th[8] = {1.0, 0, 0, 0, 0, 0, 0, 0};
  cudaMemcpy(m->thermo, th, sizeof(th), cudaMemcpyHostToDevice);
  cudaMemset(m->maxd2, 0, sizeof(unsigned int));
  *out = m;
  return MDRT_NB_OK;
}

int32_t mdrtMdDestroy(mdrtMd *m) {
  if (m) {
    cudaSetDevice(m->nb->device);
    md_free(m);
  }
  return MDRT_NB_OK;
}

int32_t mdrtMdSetThermostat(mdrtMd *m, double temperature, double tau, uint64_t seed) {
  if (!m || !(temperature >= 0)) return MDRT_NB_INVALID_ARGUMENT;
  m->temperature = temperature;
  m->tau = tau;
  m->seed = seed;
  if (m->exec) {  // parameters are baked into the graph
    cudaGraphExecDestroy(m->exec);
    cudaGraphDestroy(m->graph);
    m->exec = nullptr;
    m->graph = nullptr;
  }
  return MDRT_NB_OK;
}

// A build at x that also resets the reference positions of the test of validity.
int32_t mdrtMdBuild(mdrtMd *m, const double *x, const double box[3], void *stream) {
  if (!m || !x || !box) return MDRT_NB_INVALID_ARGUMENT;
  int32_t sizes[NB_SIZE_COUNT];
  int32_t s = mdrtNbBuild(m->handle, x, m->n, box, 0.0, stream, sizes);
  if (s) return s;
  cudaStream_t st = (cudaStream_t)stream;
  md_after_build<<<blocks_for(3 * m->n, 256), 256, 0, st>>>(3 * m->n, x, m->x_ref, m->maxd2, m->thermo,
                                                           m->nb->sizes, m->nb->status);
  return cudaGetLastError() == cudaSuccess ? MDRT_NB_OK : MDRT_NB_CUDA_ERROR;
}

int32_t mdrtMdRun(mdrtMd *m, double *x, double *v, const double box[3], double dt, int64_t steps,
                  int32_t unroll, void *stream) {
  if (!m || !x || !v || !box || !(dt > 0) || steps < 0) return MDRT_NB_INVALID_ARGUMENT;
  NbCtx &c = *m->nb;
  if (!c.built) return MDRT_NB_NOT_BUILT;
  cudaSetDevice(c.device);
  cudaStream_t st = (cudaStream_t)stream;
  if (unroll <= 0) {
    // step by step, the host reading the test of validity after each step
    int *flag = nullptr;
    if (cudaMalloc(&flag, sizeof(int)) != cudaSuccess) return MDRT_NB_CUDA_ERROR;
    int h_flag = 0;
    for (int64_t k = 0; k < steps; ++k) {
      md_step_body(*m, x, v, box, dt, st, 0, 0, flag);
      cudaMemcpyAsync(&h_flag, flag, sizeof(int), cudaMemcpyDeviceToHost, st);
      cudaStreamSynchronize(st);
      if (h_flag) {
        int32_t s = mdrtMdBuild(m, x, box, stream);
        if (s) {
          cudaFree(flag);
          return s;
        }
      }
    }
    cudaFree(flag);
    return cudaGetLastError() == cudaSuccess ? MDRT_NB_OK : MDRT_NB_CUDA_ERROR;
  }
  // a graph of `unroll` steps, each ending in a conditional rebuild
  int64_t key = c.groups_cap * 1000003 + c.list_cap * 7 + c.units_cap;
  bool stale = !m->exec || m->gx != x || m->gv != v || m->gdt != dt || m->gunroll != unroll ||
               m->gbox[0] != box[0] || m->gbox[1] != box[1] || m->gbox[2] != box[2] || m->gcap_key != key;
  if (stale) {
    if (m->exec) cudaGraphExecDestroy(m->exec);
    if (m->graph) cudaGraphDestroy(m->graph);
    m->exec = nullptr;
    m->graph = nullptr;
    cudaStream_t cap;
    cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
    cudaStream_t body;
    cudaStreamCreateWithFlags(&body, cudaStreamNonBlocking);
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return MDRT_NB_CUDA_ERROR;
    m->handles.assign(unroll, 0);
    for (int k = 0; k < unroll && e == cudaSuccess; ++k) {
      cudaStreamCaptureStatus status;
      cudaGraph_t g;
      const cudaGraphNode_t *deps = nullptr;
      size_t ndeps = 0;
      e = cudaStreamGetCaptureInfo(cap, &status, nullptr, &g, &deps, &ndeps);
      if (e != cudaSuccess) break;
      e = cudaGraphConditionalHandleCreate(&m->handles[k], g, 0, cudaGraphCondAssignDefault);
      if (e != cudaSuccess) break;
      md_step_body(*m, x, v, box, dt, cap, m->handles[k], 1, nullptr);
      e = cudaStreamGetCaptureInfo(cap, &status, nullptr, &g, &deps, &ndeps);
      if (e != cudaSuccess) break;
      cudaGraphNodeParams cp = {};
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = m->handles[k];
      cp.conditional.type = cudaGraphCondTypeIf;
      cp.conditional.size = 1;
      cudaGraphNode_t node;
      e = cudaGraphAddNode(&node, g, deps, ndeps, &cp);
      if (e != cudaSuccess) break;
      e = cudaStreamUpdateCaptureDependencies(cap, &node, 1, cudaStreamSetCaptureDependencies);
      if (e != cudaSuccess) break;
      cudaGraph_t bodyGraph = cp.conditional.phGraph_out[0];
      e = cudaStreamBeginCaptureToGraph(body, bodyGraph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) break;
      md_rebuild_body(*m, x, box, body);
      e = cudaStreamEndCapture(body, nullptr);
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
    e = cudaGraphInstantiate(&m->exec, graph, 0);
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
  int64_t launches = steps / unroll;
  for (int64_t k = 0; k < launches; ++k)
    if (cudaGraphLaunch(m->exec, st) != cudaSuccess) return MDRT_NB_CUDA_ERROR;
  int64_t rest = steps - launches * unroll;
  if (rest > 0) return mdrtMdRun(m, x, v, box, dt, rest, 0, stream);
  return cudaGetLastError() == cudaSuccess ? MDRT_NB_OK : MDRT_NB_CUDA_ERROR;
}

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
  return MDRT_NB_OK;
}

// The forces of the last step (device f64 [n, 3]).
int32_t mdrtMdForces(mdrtMd *m, double **forces) {
  if (!m || !forces) return MDRT_NB_INVALID_ARGUMENT;
  *forces = m->force;
  return MDRT_NB_OK;
}

}  // extern "C"
