// Core definitions shared by every LBM kernel: lattice tables as compile-time
// constants, population storage codecs, the device view of one scene, and the
// FP64 sphere helpers (contains / surfaceVelocity / impulse) evaluated without
// FMA contraction so the solid mask is bit-exact against the reference's
// JavaScript doubles.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>
#include <utility>

#include "lbm_b200.h"

namespace lbm {

constexpr int Q27 = 27;
constexpr int Q7 = 7;
constexpr uint8_t TAG_FLUID = 0;
constexpr uint8_t TAG_SOLID = 1;
constexpr uint8_t TAG_WALL = 2;

// D3Q27 velocity set in opposite pairs, rest first (src/lattices.js:34-49);
// the first seven entries double as the D3Q7 set (src/lattices.js:79-84).
constexpr int kDir[27][3] = {
    {0, 0, 0},   {1, 0, 0},   {-1, 0, 0}, {0, 1, 0},   {0, -1, 0},  {0, 0, 1},   {0, 0, -1},
    {1, 1, 0},   {-1, -1, 0}, {1, -1, 0}, {-1, 1, 0},  {1, 0, 1},   {-1, 0, -1}, {1, 0, -1},
    {-1, 0, 1},  {0, 1, 1},   {0, -1, -1}, {0, 1, -1}, {0, -1, 1},  {1, 1, 1},   {-1, -1, -1},
    {1, 1, -1},  {-1, -1, 1}, {1, -1, 1}, {-1, 1, -1}, {-1, 1, 1},  {1, -1, -1}};

template <int K>
struct D27 {
  static constexpr int ex = kDir[K][0];
  static constexpr int ey = kDir[K][1];
  static constexpr int ez = kDir[K][2];
  static constexpr int nnz = (ex != 0) + (ey != 0) + (ez != 0);
  // Float32Array weights: the double 8/27, 2/27, 1/54, 1/216 rounded to float
  // (src/lattices.js:22, 52-57).
  static constexpr float w = (float)(nnz == 0   ? 8.0 / 27.0
                                     : nnz == 1 ? 2.0 / 27.0
                                     : nnz == 2 ? 1.0 / 54.0
                                                : 1.0 / 216.0);
  static constexpr int opp = K == 0 ? 0 : ((K & 1) ? K + 1 : K - 1);  // lattices.js:66-69
};

template <int K>
struct D7 {
  static constexpr int ex = kDir[K][0];
  static constexpr int ey = kDir[K][1];
  static constexpr int ez = kDir[K][2];
  static constexpr float w = (float)(K == 0 ? 0.25 : 0.125);  // lattices.js:85
  static constexpr int opp = K == 0 ? 0 : ((K & 1) ? K + 1 : K - 1);
};

// Runtime-indexable copy for kernels that loop over directions at run time.
static __constant__ signed char c_dir[27][3] = {
    {0, 0, 0},   {1, 0, 0},   {-1, 0, 0}, {0, 1, 0},   {0, -1, 0},  {0, 0, 1},   {0, 0, -1},
    {1, 1, 0},   {-1, -1, 0}, {1, -1, 0}, {-1, 1, 0},  {1, 0, 1},   {-1, 0, -1}, {1, 0, -1},
    {-1, 0, 1},  {0, 1, 1},   {0, -1, -1}, {0, 1, -1}, {0, -1, 1},  {1, 1, 1},   {-1, -1, -1},
    {1, 1, -1},  {-1, -1, 1}, {1, -1, 1}, {-1, 1, -1}, {-1, 1, 1},  {1, -1, -1}};

__host__ __device__ inline int dcomp(int k, int a) {
#ifdef __CUDA_ARCH__
  return c_dir[k][a];
#else
  return kDir[k][a];
#endif
}

template <int B, int E, class F>
__device__ __forceinline__ void static_for(F &&f) {
  if constexpr (B < E) {
    f(std::integral_constant<int, B>{});
    static_for<B + 1, E>(f);
  }
}

// ---------------------------------------------------------------- explicit rounding
// Arithmetic that must give the same bits wherever it is inlined (the fused
// collision runs for tile cells and for halo cells of neighbouring tiles):
// each operation rounds once and the compiler may not contract or reorder it.
// FP32: mul / add / sub round to nearest, rfma is one fused multiply-add.
// FP64: rfma is a multiply then an add (the FP64 form follows the reference's
// unfused double arithmetic).
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float rfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rfma(double a, double b, double c) { return __dadd_rn(__dmul_rn(a, b), c); }

// ---------------------------------------------------------------- storage codecs
// FP32/FP64 store raw populations.  FP16/BF16 store the offset from a
// reference value: w_k for f, w_k * phi(cell) for h, so the stored numbers are
// small and keep their relative precision.
template <class S>
struct Codec;

// enc4: one cell's group of four values at once, element for element what
// enc gives (the 16-bit forms convert pairs with one packing conversion, each
// element rounded to nearest even as by the scalar conversion).
template <>
struct Codec<float> {
  static constexpr bool offset = false;
  __device__ __forceinline__ static float dec(float v, float) { return v; }
  __device__ __forceinline__ static float enc(float v, float) { return v; }
  __device__ __forceinline__ static void enc4(const float (&v)[4], const float (&)[4], float (&o)[4]) {
    o[0] = v[0], o[1] = v[1], o[2] = v[2], o[3] = v[3];
  }
};
template <>
struct Codec<double> {
  static constexpr bool offset = false;
  __device__ __forceinline__ static double dec(double v, double) { return v; }
  __device__ __forceinline__ static double enc(double v, double) { return v; }
  __device__ __forceinline__ static void enc4(const double (&v)[4], const double (&)[4], double (&o)[4]) {
    o[0] = v[0], o[1] = v[1], o[2] = v[2], o[3] = v[3];
  }
};
template <>
struct Codec<__half> {
  static constexpr bool offset = true;
  __device__ __forceinline__ static float dec(__half v, float ref) { return __fadd_rn(__half2float(v), ref); }
  __device__ __forceinline__ static __half enc(float v, float ref) { return __float2half_rn(__fsub_rn(v, ref)); }
  __device__ __forceinline__ static void enc4(const float (&v)[4], const float (&r)[4], __half (&o)[4]) {
    const __half2 a = __floats2half2_rn(__fsub_rn(v[0], r[0]), __fsub_rn(v[1], r[1]));
    const __half2 b = __floats2half2_rn(__fsub_rn(v[2], r[2]), __fsub_rn(v[3], r[3]));
    o[0] = __low2half(a), o[1] = __high2half(a), o[2] = __low2half(b), o[3] = __high2half(b);
  }
};
template <>
struct Codec<__nv_bfloat16> {
  static constexpr bool offset = true;
  __device__ __forceinline__ static float dec(__nv_bfloat16 v, float ref) {
    return __fadd_rn(__bfloat162float(v), ref);
  }
  __device__ __forceinline__ static __nv_bfloat16 enc(float v, float ref) {
    return __float2bfloat16_rn(__fsub_rn(v, ref));
  }
  __device__ __forceinline__ static void enc4(const float (&v)[4], const float (&r)[4],
                                              __nv_bfloat16 (&o)[4]) {
    const __nv_bfloat162 a = __floats2bfloat162_rn(__fsub_rn(v[0], r[0]), __fsub_rn(v[1], r[1]));
    const __nv_bfloat162 b = __floats2bfloat162_rn(__fsub_rn(v[2], r[2]), __fsub_rn(v[3], r[3]));
    o[0] = __low2bfloat16(a), o[1] = __high2bfloat16(a), o[2] = __low2bfloat16(b), o[3] = __high2bfloat16(b);
  }
};

// ---------------------------------------------------------------- population layout
// Populations are stored in blocks of 8 consecutive cells (flat cell order).
// Inside a block the directions form groups of four (the last group padded),
// and a cell's four values of a group are adjacent: element (k, i) of a
// Q-direction lattice is at
//   ((i >> 3) * G + (k >> 2)) * 32 + (i & 7) * 4 + (k & 3),   G = (Q + 3) / 4.
// One cell's group is a single 16-byte (FP32) or 8-byte (FP16/BF16) vector,
// and a warp reading one group of 32 consecutive cells reads whole lines.
template <int Q>
struct PopGroups {
  static constexpr int G = (Q + 3) / 4;  // groups per cell
  static constexpr int BLOCK = 32 * G;   // elements per 8-cell block
};
// offset of direction k inside its cell's part of a block
__host__ __device__ __forceinline__ constexpr int pofs(int k) { return (k >> 2) * 32 + (k & 3); }
template <int Q>
__host__ __device__ __forceinline__ long long pidx(int k, long long i) {
  return (i >> 3) * PopGroups<Q>::BLOCK + (i & 7) * 4 + pofs(k);
}
// elements of tail pad after every macro and tag array: the pipelined step
// copies rows rounded out to 16-byte units, which can reach past the last cell
constexpr long long ARRAY_PAD = 64;

// elements of a Q-direction lattice over n cells (whole blocks)
__host__ __device__ inline long long pop_elems(long long n, int Q) { return (n + 7) / 8 * 32 * ((Q + 3) / 4); }

// ---------------------------------------------------------------- scene view
// Device pointers of one scene.  Index c in [0,1] selects a ping-pong half:
// populations and macros are double-buffered so the fused step can read the
// current half (including neighbours owned by other CTAs) while writing the
// next.  Macro type is Real (float, or double for the FP64 form).
template <class PopT, class Real>
struct Scene {
  int nx, ny, nz;
  long long n;  // cells
  PopT *F[2];
  PopT *H[2];
  Real *phi[2], *rho[2], *ux[2], *uy[2], *uz[2];
  uint8_t *tag, *tagPrev;
  // phase-by-phase scratch (allocated on first use)
  Real *gx, *gy, *gz, *lap;
  Real *usx, *usy, *usz;
  Real *bfx, *bfy, *bfz;  // body force; null when never set

  // Where ux and uy live.  When a population is as wide as a macro (FP32 and
  // FP64 storage) they take the pad slots of the last direction group of f
  // (element 27) and of h (element 7), which every step reads and writes with
  // their groups anyway, so the step moves 16 B (FP32) less per cell than
  // with separate arrays; the 16-bit forms keep the ux, uy arrays.  Every
  // access goes through these four functions.
  static constexpr bool UPAD = sizeof(PopT) == sizeof(Real);
  __device__ __forceinline__ Real ux_at(int c, long long i) const {
    if constexpr (UPAD) return (Real)F[c][pidx<27>(27, i)];
    else return ux[c][i];
  }
  __device__ __forceinline__ Real uy_at(int c, long long i) const {
    if constexpr (UPAD) return (Real)H[c][pidx<7>(7, i)];
    else return uy[c][i];
  }
  __device__ __forceinline__ void set_ux(int c, long long i, Real v) const {
    if constexpr (UPAD) F[c][pidx<27>(27, i)] = (PopT)v;
    else ux[c][i] = v;
  }
  __device__ __forceinline__ void set_uy(int c, long long i, Real v) const {
    if constexpr (UPAD) H[c][pidx<7>(7, i)] = (PopT)v;
    else uy[c][i] = v;
  }
};

// Scalar physics parameters, precomputed on the host in double
// (src/sim.js:327-331, 410-416, 490-492).
struct StepConst {
  double tau, tauPhi, sigma, gravity, rhoL, rhoG, W;
  double invTau, invTauPhi, beta, kappa, dRho, A, sharpC;
};

inline StepConst make_const(const lbm_params &p) {
  StepConst c;
  c.tau = p.tau;
  c.tauPhi = p.tauPhi;
  c.sigma = p.sigma;
  c.gravity = p.gravity;
  c.rhoL = p.rhoL;
  c.rhoG = p.rhoG;
  c.W = p.W;
  c.invTau = 1 / p.tau;
  c.invTauPhi = 1 / p.tauPhi;
  c.beta = 12 * p.sigma / p.W;
  c.kappa = 1.5 * p.sigma * p.W;
  c.dRho = p.rhoL - p.rhoG;
  c.A = (1 - 0.5 * c.invTau) * 3.0;
  double Mphi = 0.25 * (p.tauPhi - 0.5);
  double guoHalf = 1.0 - 0.5 * c.invTauPhi;
  c.sharpC = 4.0 * Mphi * guoHalf / p.W;
  return c;
}

// ---------------------------------------------------------------- FP64 sphere math
// Evaluated with explicit round-to-nearest intrinsics (no contraction) in the
// reference's evaluation order.
struct SphereDesc {
  double cx, cy, cz, r, vx, vy, vz, wx, wy, wz;
};

__device__ __forceinline__ bool sphere_contains(const SphereDesc &b, int x, int y, int z) {
  // src/solid.js:50-55
  double dx = __dsub_rn(__dadd_rn((double)x, 0.5), b.cx);
  double dy = __dsub_rn(__dadd_rn((double)y, 0.5), b.cy);
  double dz = __dsub_rn(__dadd_rn((double)z, 0.5), b.cz);
  double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
  return d2 <= __dmul_rn(b.r, b.r);
}

__device__ __forceinline__ void sphere_surface_velocity(const SphereDesc &b, int x, int y, int z,
                                                        double &ox, double &oy, double &oz) {
  // src/solid.js:57-66
  double rx = __dsub_rn(__dadd_rn((double)x, 0.5), b.cx);
  double ry = __dsub_rn(__dadd_rn((double)y, 0.5), b.cy);
  double rz = __dsub_rn(__dadd_rn((double)z, 0.5), b.cz);
  ox = __dadd_rn(b.vx, __dsub_rn(__dmul_rn(b.wy, rz), __dmul_rn(b.wz, ry)));
  oy = __dadd_rn(b.vy, __dsub_rn(__dmul_rn(b.wz, rx), __dmul_rn(b.wx, rz)));
  oz = __dadd_rn(b.vz, __dsub_rn(__dmul_rn(b.wx, ry), __dmul_rn(b.wy, rx)));
}

// Torque arm and increments of applyImpulseAtCell (src/solid.js:70-80).
__device__ __forceinline__ void impulse_terms(const SphereDesc &b, int x, int y, int z, double px,
                                              double py, double pz, double acc[6]) {
  double rx = __dsub_rn(__dadd_rn((double)x, 0.5), b.cx);
  double ry = __dsub_rn(__dadd_rn((double)y, 0.5), b.cy);
  double rz = __dsub_rn(__dadd_rn((double)z, 0.5), b.cz);
  acc[0] = __dadd_rn(acc[0], px);
  acc[1] = __dadd_rn(acc[1], py);
  acc[2] = __dadd_rn(acc[2], pz);
  acc[3] = __dadd_rn(acc[3], __dsub_rn(__dmul_rn(ry, pz), __dmul_rn(rz, py)));
  acc[4] = __dadd_rn(acc[4], __dsub_rn(__dmul_rn(rz, px), __dmul_rn(rx, pz)));
  acc[5] = __dadd_rn(acc[5], __dsub_rn(__dmul_rn(rx, py), __dmul_rn(ry, px)));
}

// Composite-solid owner: first sphere containing the cell, -1 for none.
template <int MAXS>
__device__ __forceinline__ int owner_of(const SphereDesc *sph, int nsph, int x, int y, int z) {
  for (int b = 0; b < nsph && b < MAXS; b++)
    if (sphere_contains(sph[b], x, y, z)) return b;
  return -1;
}

// Integer bounding box of the cells a sphere can contain (centre +0.5 test):
// x + 0.5 in [cx - r, cx + r]  =>  x in [ceil(cx - r - 0.5), floor(cx + r - 0.5)].
struct Box {
  int lo[3], hi[3];  // inclusive; empty when lo > hi
};

__host__ __device__ inline Box sphere_box(double cx, double cy, double cz, double r, int nx, int ny,
                                          int nz) {
  Box b;
  double c[3] = {cx, cy, cz};
  int n[3] = {nx, ny, nz};
  for (int a = 0; a < 3; a++) {
    double lo = c[a] - r - 0.5, hi = c[a] + r - 0.5;
    // one cell of slack on each side against rounding at the boundary
    long long l = (long long)floor(lo) - 1, h = (long long)floor(hi) + 1;
    if (!(lo == lo) || !(hi == hi)) {  // NaN centre: cover nothing
      l = 1;
      h = 0;
    }
    if (l < 1) l = 1;
    if (h > n[a] - 2) h = n[a] - 2;
    b.lo[a] = (int)l;
    b.hi[a] = (int)h;
  }
  return b;
}

__host__ __device__ inline bool box_empty(const Box &b) {
  return b.lo[0] > b.hi[0] || b.lo[1] > b.hi[1] || b.lo[2] > b.hi[2];
}

__host__ __device__ inline Box box_union(const Box &a, const Box &b) {
  if (box_empty(a)) return b;
  if (box_empty(b)) return a;
  Box u;
  for (int d = 0; d < 3; d++) {
    u.lo[d] = a.lo[d] < b.lo[d] ? a.lo[d] : b.lo[d];
    u.hi[d] = a.hi[d] > b.hi[d] ? a.hi[d] : b.hi[d];
  }
  return u;
}

__host__ __device__ inline Box box_grow(const Box &a, int g, int nx, int ny, int nz) {
  if (box_empty(a)) return a;
  Box u;
  int n[3] = {nx, ny, nz};
  for (int d = 0; d < 3; d++) {
    u.lo[d] = a.lo[d] - g < 0 ? 0 : a.lo[d] - g;
    u.hi[d] = a.hi[d] + g > n[d] - 1 ? n[d] - 1 : a.hi[d] + g;
  }
  return u;
}

__host__ __device__ inline long long box_cells(const Box &b) {
  if (box_empty(b)) return 0;
  return (long long)(b.hi[0] - b.lo[0] + 1) * (b.hi[1] - b.lo[1] + 1) * (b.hi[2] - b.lo[2] + 1);
}

// Impulse accumulation target of one sphere: a dense array of 6 doubles per
// cell over the sphere's bounding box grown by one cell.  Each fluid cell's
// slot is written only by the thread that owns the cell, so the result does not
// depend on tiling or scheduling; a fixed-order reduction sums it.
struct ImpulseTarget {
  double *acc;  // [cells][6]
  int lo[3], dim[3];
};

struct SolidSet {
  int nsph;
  // z slab: dead cells outside local planes [zlo, zend) give no impulse (their
  // slab's neighbour owns them); zend = 0 (the default) means no limit
  int zlo, zend;
  SphereDesc sph[LBM_MAX_SPHERES];
  ImpulseTarget imp[LBM_MAX_SPHERES];
};

// Per-step plan of the sparse work around the spheres, in device memory.  The
// host-driven API computes it on the host and copies it up; the device-resident
// loop computes it with k_plan from the device copy of the sphere state.  Every
// kernel of a step reads it, so launch grids can be sized by upper bounds.
struct Plan {
  SolidSet ss;
  Box U;             // retag / fresh-dead compaction box
  long long ucells;  // cells in U
  int nchunks;       // compaction chunks of U
  int redChunks;     // impulse-reduction chunks (max over spheres)
  long long impDoubles;
  Box boxLast, boxLastLast;  // sphere boxes of the two previous retags
  int fullRetag;             // retag the whole grid for this many more steps
  int overflow;              // the plan exceeded the launch capacity
};


}  // namespace lbm
