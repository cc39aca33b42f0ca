// The fused LBM step kernel (one launch per step over the whole grid).
//
// A CTA owns a 32 x TY column of cells and marches it up a range of z planes,
// with TY "cell" warps (one cell per thread) and two "halo" warps.  For each
// plane z:
//   1. plane z+1 is collided: every cell thread loads its cell's 27 + 7
//      populations, phi stencil, rho and u, evaluates the reference's BGK
//      collisions (collideHydro src/sim.js:406-464, collidePhase
//      src/sim.js:324-364) in registers and, after a barrier that ends the
//      previous plane's pull, writes the post-collision values into a
//      shared-memory ring; meanwhile the halo warps collide the
//      one-cell in-plane halo, only for the directions that point into the
//      tile (halo warp A: the rows above and below, halo warp B: the side
//      columns and corners);
//   2. after a barrier the cell threads pull plane z from the ring
//      (streamPhase src/sim.js:376-397, streamHydroAndMacro src/sim.js:509-543):
//      fluid sources give their post-collision value, wall and solid sources
//      bounce back the cell's own value, SOLID sources add the Ladd
//      moving-wall term and FP64 momentum exchange; then the macros
//      (src/sim.js:545-576), and the new populations and macros are written
//      once.
//
// The collision is evaluated in the equivalent form
//   f*_k = (1 - w) f_k + w_k (C0 + e.V + (e.u)(e.Q)),
//   C0 = w sumF - 1.5 w rho_phase u^2 - A u.F,  V = 3 w rho_phase u + A F,
//   Q  = 4.5 w rho_phase u + 3 A F   (w = 1/tau, A = 3(1 - w/2)),
//   h*_k = (1 - wp) h_k + w7_k (wp phi + e.(4 wp phi u + S)),
// which expands to the reference's feq / Guo source / sharpening terms.
//
// Ring layout: directions grouped by e_z.  Values pulled from plane z+1
// (e_z = -1) are read in the iteration they are written, but a plane's own
// e_z = -1 values are needed for bounce-back, so that group keeps 2 planes;
// e_z = 0 keeps 2 planes; e_z = +1 keeps 3.
//
// Per cell and step the kernel reads the 34 populations, phi, rho, u and the
// tag once and writes 34 populations and 5 macros once (313 B at FP32).
#pragma once

#include "lbm_kernels.cuh"

namespace lbm {

// An encoded tensor map (the driver's 128-byte, 64-byte aligned descriptor).
struct alignas(64) TensorMap {
  unsigned long long w[16];
};
// Tensor maps of one scene for the TMA-staged form (tiles of TMA_ROWS rows):
// per half, the f and h populations as 4-D arrays (elements of an 8-cell
// block, blocks of a row, y, z; box: 4 blocks x TMA_ROWS rows) and phi, rho,
// ux, uy, uz as 3-D arrays (x, y, z; box 32 x TMA_ROWS, phi 40 x
// TMA_ROWS + 2); the tags (x, y, z; box 32 x TMA_ROWS).  Built on the host
// when the scene is created, for nx a multiple of 16.
constexpr int TMA_ROWS = 6;
struct StageMaps {
  TensorMap f[2], h[2], phi[2], rho[2], ux[2], uy[2], uz[2], tag;
};

template <class PopT>
struct FusedArgs {
  Scene<PopT, typename Prec<PopT>::Real> s;
  int cur;
  int zchunk;
  double om, omP, A, beta4, kappa, rhoG, dRho, gravity, sharpC4;
  const SolidSet *ss;
  int *status;   // set non-zero when a bounded wait of the step runs out
  int withhold;  // test hook: the bulk-staged form does not issue each tile's first copy
  uint8_t *pack; // frame step: the RG8 volume of the step's result (planes 1 .. nz-2), else null
  const StageMaps *maps;  // tensor maps of the TMA-staged form (device memory), else null
};

// slot of direction k within its e_z group (0..8 for D3Q27)
constexpr int slot27(int k) {
  int s = 0;
  for (int j = 0; j < k; j++)
    if (kDir[j][2] == kDir[k][2]) s++;
  return s;
}
// the same, indexable at run time
static __constant__ signed char c_slot27[27] = {0, 1, 2, 3, 4, 0, 0, 5, 6, 7, 8, 1, 1, 2,
                                                 2, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 8, 8};
// ring plane offsets (in planes of NC values)
constexpr int RING_F_M = 0, RING_F_Z = 18, RING_F_P = 36;  // 2x9, 2x9, 3x9
constexpr int RING_H_M = 63, RING_H_Z = 65, RING_H_P = 75;  // 2x1, 2x5, 3x1
constexpr int RING_PLANES = 78;

// Shared memory of one CTA: the post-collision ring (78 planes of the
// halo-padded tile) and the tags of three planes.
template <class PopT, int TY>
struct FusedSmem {
  using Real = typename Prec<PopT>::Real;
  static constexpr int RX = 34, RY = TY + 2, NC = RX * RY;
  static constexpr size_t ringBytes = (size_t)RING_PLANES * NC * sizeof(Real);
  static constexpr size_t bytes = ringBytes + 3 * NC;
  static constexpr int warps = TY + 2;  // TY cell warps, 2 halo warps
  static constexpr int threads = 32 * warps;
};

// CTAs per SM the register budget is sized for
template <class PopT, int TY>
struct FusedOcc {
  static constexpr int blocks = TY >= 8 ? 2 : (TY >= 4 ? 3 : 5);
};

// ---------------------------------------------------------------- bulk copies
// cp.async.bulk global -> shared with an mbarrier counting the bytes.  Every
// wait is bounded (LBM_STAGE_WAIT_NS of %globaltimer); a wait that runs out
// returns false and the caller records the fault and stops the tile.
#ifndef LBM_STAGE_WAIT_NS
#define LBM_STAGE_WAIT_NS 1000000000ull
#endif
// a wait also needs this many polls before it gives up, so time during which
// the context was not running does not count as waiting
#ifndef LBM_STAGE_WAIT_POLLS
#define LBM_STAGE_WAIT_POLLS 65536u
#endif
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint32_t bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_init_count(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_inval(uint32_t bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}
// One box of a tensor map (a 3-D or 4-D array in global memory) into shared
// memory, completion counted in bytes on an mbarrier.  Coordinates are
// innermost first; the innermost one times the element size is a multiple of
// 16 bytes, the destination is 128-byte aligned, and cells of the box outside
// the array arrive as zeros (the whole box is counted).  No multicast.
__device__ __forceinline__ void tma_g2s_3d(uint32_t dst, const void *map, int c0, int c1, int c2, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void tma_g2s_4d(uint32_t dst, const void *map, int c0, int c1, int c2, int c3,
                                           uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
      : "memory");
}
// One box of a tensor map brought into L2 only (no shared memory, no
// completion to wait for); the same coordinate rules as the copies above,
// and the parts of the box outside the array are skipped.  No multicast.
__device__ __forceinline__ void tma_l2_3d(const void *map, int c0, int c1, int c2) {
  asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];" ::"l"(map), "r"(c0),
               "r"(c1), "r"(c2)
               : "memory");
}
__device__ __forceinline__ void tma_l2_4d(const void *map, int c0, int c1, int c2, int c3) {
  asm volatile("cp.async.bulk.prefetch.tensor.4d.L2.global.tile [%0, {%1, %2, %3, %4}];" ::"l"(map), "r"(c0),
               "r"(c1), "r"(c2), "r"(c3)
               : "memory");
}
// orders this CTA's earlier shared-memory reads before later copies of the
// asynchronous proxy into the same bytes
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// Per-thread asynchronous copies global -> shared (cp.async, 4 / 8 / 16
// bytes, both addresses aligned to the size).  A thread's copies complete, and
// become visible to that thread, at its next cp_async_wait_all; the 16-byte
// form keeps the line in L2 only.
template <int BYTES>
__device__ __forceinline__ void cp_async(uint32_t dst, const void *src) {
  static_assert(BYTES == 4 || BYTES == 8 || BYTES == 16, "cp.async sizes");
  if constexpr (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(dst), "l"(src), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (uint32_t polls = 0;; polls++) {
    if (mbar_try(bar, parity)) return true;
    if (polls >= LBM_STAGE_WAIT_POLLS && global_ns() - t0 > LBM_STAGE_WAIT_NS) return false;
  }
}

// Directions a halo cell must collide: those pointing into the tile.
// SX / SY = +-1 select e_x / e_y equal to that value, 0 means any.
template <int SX, int SY, int K>
constexpr bool halo_dir() {
  return (SX == 0 || kDir[K][0] == SX) && (SY == 0 || kDir[K][1] == SY);
}

// does direction group g (directions 4g .. 4g+3) hold a direction a halo cell
// of side (SX, SY) needs?
template <int SX, int SY, int Q, int G>
constexpr bool halo_group() {
  for (int k = 4 * G; k < 4 * G + 4 && k < Q; k++)
    if ((SX == 0 || kDir[k][0] == SX) && (SY == 0 || kDir[k][1] == SY)) return true;
  return false;
}

template <int V>
using IC = std::integral_constant<int, V>;

// ---------------------------------------------------------------- checked build
// Built with -DLBM_CHECKED, every global and shared access of the fused kernel
// is bounds-checked; the first violation is recorded (location code, index,
// block, thread) in lbm_fault_word and the access is skipped instead of
// faulting.  Without the macro the helpers are plain loads and stores.
static __device__ unsigned long long lbm_fault_word[4];

__device__ __forceinline__ bool lbm_ok(bool ok, int code, long long idx) {
#ifdef LBM_CHECKED
  if (!ok) {
    if (atomicCAS(&lbm_fault_word[0], 0ull, (unsigned long long)code) == 0ull) {
      lbm_fault_word[1] = (unsigned long long)idx;
      lbm_fault_word[2] = blockIdx.x | ((unsigned long long)blockIdx.y << 20) |
                          ((unsigned long long)blockIdx.z << 40);
      lbm_fault_word[3] = threadIdx.x | (threadIdx.y << 8);
    }
  }
  return ok;
#else
  (void)code;
  (void)idx;
  return true;
#endif
}

// Location code recorded when a bounded wait for a staged plane runs out.
constexpr int FAULT_STAGE_WAIT = 90;
__device__ __forceinline__ void record_stage_timeout(int q) {
  if (atomicCAS(&lbm_fault_word[0], 0ull, (unsigned long long)FAULT_STAGE_WAIT) == 0ull) {
    lbm_fault_word[1] = (unsigned long long)q;
    lbm_fault_word[2] = blockIdx.x | ((unsigned long long)blockIdx.y << 20) |
                        ((unsigned long long)blockIdx.z << 40);
    lbm_fault_word[3] = threadIdx.x | (threadIdx.y << 8);
  }
}

template <class T>
__device__ __forceinline__ T ldg_at(const T *p, long long idx, long long lim, int code) {
  if (!lbm_ok(idx >= 0 && idx < lim, code, idx)) return T();
  return __ldg(p + idx);
}
template <class T>
__device__ __forceinline__ void st_at(T *p, long long idx, long long lim, int code, T v) {
  if (lbm_ok(idx >= 0 && idx < lim, code, idx)) p[idx] = v;
}
__device__ __forceinline__ int sm_at(int idx, int lim, int code) {
  return lbm_ok(idx >= 0 && idx < lim, code, idx) ? idx : 0;
}

// One cell's group of four populations (adjacent and aligned to the group's
// size): one 16-byte access for FP32, 8 bytes for FP16/BF16, two 16-byte
// accesses for FP64.
template <class PopT>
__device__ __forceinline__ void ld4_global(const PopT *p, PopT (&o)[4]) {
  if constexpr (sizeof(PopT) == 4) {
    const float4 t = __ldg(reinterpret_cast<const float4 *>(p));
    memcpy(o, &t, 16);
  } else if constexpr (sizeof(PopT) == 8) {
    const double2 a = __ldg(reinterpret_cast<const double2 *>(p));
    const double2 b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
    memcpy(o, &a, 16);
    memcpy(o + 2, &b, 16);
  } else {
    const uint2 t = __ldg(reinterpret_cast<const uint2 *>(p));
    memcpy(o, &t, 8);
  }
}
template <class PopT>
__device__ __forceinline__ void ld4_shared(const PopT *p, PopT (&o)[4]) {
  if constexpr (sizeof(PopT) == 4) {
    const float4 t = *reinterpret_cast<const float4 *>(p);
    memcpy(o, &t, 16);
  } else if constexpr (sizeof(PopT) == 8) {
    const double2 a = reinterpret_cast<const double2 *>(p)[0];
    const double2 b = reinterpret_cast<const double2 *>(p)[1];
    memcpy(o, &a, 16);
    memcpy(o + 2, &b, 16);
  } else {
    const uint2 t = *reinterpret_cast<const uint2 *>(p);
    memcpy(o, &t, 8);
  }
}
template <class PopT>
__device__ __forceinline__ void st4_global(PopT *p, const PopT (&v)[4]) {
  if constexpr (sizeof(PopT) == 4) {
    float4 t;
    memcpy(&t, v, 16);
    *reinterpret_cast<float4 *>(p) = t;
  } else if constexpr (sizeof(PopT) == 8) {
    double2 a, b;
    memcpy(&a, v, 16);
    memcpy(&b, v + 2, 16);
    reinterpret_cast<double2 *>(p)[0] = a;
    reinterpret_cast<double2 *>(p)[1] = b;
  } else {
    uint2 t;
    memcpy(&t, v, 8);
    *reinterpret_cast<uint2 *>(p) = t;
  }
}
// bounds-checked forms (group of elements idx .. idx + 3); a load that is not
// wanted or out of range gives zeros
template <class PopT>
__device__ __forceinline__ void ldg4_at(const PopT *p, long long idx, long long lim, int code, bool want,
                                        PopT (&o)[4]) {
  if (want && lbm_ok(idx >= 0 && idx + 3 < lim, code, idx)) {
    ld4_global(p + idx, o);
  } else {
    o[0] = o[1] = o[2] = o[3] = PopT();
  }
}
template <class PopT>
__device__ __forceinline__ void st4_at(PopT *p, long long idx, long long lim, int code, const PopT (&v)[4]) {
  if (lbm_ok(idx >= 0 && idx + 3 < lim, code, idx)) st4_global(p + idx, v);
}

// Everything the collision of one cell reads from global memory.
template <class PopT>
struct CellLoad {
  using Real = typename Prec<PopT>::Real;
  PopT fv[Q27];
  PopT hv[Q7];
  Real p, pxp, pxm, pyp, pym, pzp, pzm, sumF, ux, uy, uz;
  uint8_t tg;
};

// What the collision of one cell puts into the shared-memory ring: its
// post-collision populations and its tag.  Halo warp A's two cells (the rows
// above and below the tile) share one: their direction sets (e_y = +1 and
// e_y = -1) are disjoint, and the lower row's tag goes to tg2.
template <class PopT>
struct CellOut {
  using Real = typename Prec<PopT>::Real;
  Real f[Q27];
  Real h[Q7];
  uint8_t tg, tg2;
};

// Physics constants of the fused collision in the storage form's arithmetic type.
template <class Real>
struct CollK {
  Real om, omP, A, beta4, kappa, rhoG, dRho, grav, sharpC4;
};
template <class PopT>
__device__ __forceinline__ CollK<typename Prec<PopT>::Real> coll_consts(const FusedArgs<PopT> &a) {
  using Real = typename Prec<PopT>::Real;
  return CollK<Real>{(Real)a.om,   (Real)a.omP,  (Real)a.A,    (Real)a.beta4,  (Real)a.kappa,
                     (Real)a.rhoG, (Real)a.dRho, (Real)a.gravity, (Real)a.sharpC4};
}

// e.X for a lattice direction (components -1, 0, 1): signed sums, the first
// term taken exactly
template <int ex, int ey, int ez, class Real>
__device__ __forceinline__ Real edot(Real X, Real Y, Real Z) {
  Real r = 0;
  bool first = true;
  if constexpr (ex != 0) {
    r = ex > 0 ? X : -X;
    first = false;
  }
  if constexpr (ey != 0) {
    r = first ? (ey > 0 ? Y : -Y) : (ey > 0 ? radd(r, Y) : rsub(r, Y));
    first = false;
  }
  if constexpr (ez != 0) r = first ? (ez > 0 ? Z : -Z) : (ez > 0 ? radd(r, Z) : rsub(r, Z));
  return r;
}

// The collision of one cell into registers (o).  MODE 0: every direction (a
// tile cell; opposite pairs evaluated together); MODE 1: the directions of the
// compile-time halo side (SX, SY); MODE 2: every direction, one at a time (a
// halo cell whose side is known at run time).  Returns gradient, laplacian
// and phi of the cell.  Every operation rounds explicitly (rmul / radd / rsub
// / rfma), so a tile cell and a halo cell of another tile get the same bits
// whatever the compiler would contract in either context.
template <class PopT, int MODE, int SX, int SY>
__device__ __forceinline__ void collide_cell(const CollK<typename Prec<PopT>::Real> &K, const CellLoad<PopT> &L,
                                             CellOut<PopT> &o, typename Prec<PopT>::Real &ogx,
                                             typename Prec<PopT>::Real &ogy, typename Prec<PopT>::Real &ogz,
                                             typename Prec<PopT>::Real &olap, typename Prec<PopT>::Real &ophi) {
  using Real = typename Prec<PopT>::Real;
  using C = Codec<PopT>;
  if constexpr (MODE == 1 && SY < 0) o.tg2 = L.tg;
  else o.tg = L.tg;
  const Real om = K.om, omP = K.omP, A = K.A, beta4 = K.beta4, kappa = K.kappa, rhoG = K.rhoG;
  const Real dRho = K.dRho, grav = K.grav, sharpC4 = K.sharpC4;
  const Real p = L.p, ux = L.ux, uy = L.uy, uz = L.uz;
  const Real half = (Real)0.5, one = (Real)1, two = (Real)2;
  const Real gxv = rmul(half, rsub(L.pxp, L.pxm));
  const Real gyv = rmul(half, rsub(L.pyp, L.pym));
  const Real gzv = rmul(half, rsub(L.pzp, L.pzm));
  const Real lap = rfma((Real)-6, p, radd(radd(radd(radd(radd(L.pxp, L.pxm), L.pyp), L.pym), L.pzp), L.pzm));
  const Real rhoPh = rfma(p, dRho, rhoG);
  const Real mu = rfma(-kappa, lap, rmul(rmul(rmul(beta4, p), rsub(p, one)), rfma(two, p, -one)));
  const Real Fx = rmul(mu, gxv), Fy = rfma(mu, gyv, rmul(rhoPh, grav)), Fz = rmul(mu, gzv);
  const Real u2 = rfma(uz, uz, rfma(uy, uy, rmul(ux, ux)));
  const Real uF = rfma(uz, Fz, rfma(uy, Fy, rmul(ux, Fx)));
  const Real orh = rmul(om, rhoPh);
  const Real C0 = rfma(-A, uF, rfma(rmul((Real)-1.5, orh), u2, rmul(om, L.sumF)));
  const Real orh3 = rmul((Real)3, orh);
  const Real Vx = rfma(A, Fx, rmul(orh3, ux)), Vy = rfma(A, Fy, rmul(orh3, uy)), Vz = rfma(A, Fz, rmul(orh3, uz));
  const Real A3 = rmul((Real)3, A), orh45 = rmul((Real)4.5, orh);
  const Real Qx = rfma(A3, Fx, rmul(orh45, ux)), Qy = rfma(A3, Fy, rmul(orh45, uy)),
             Qz = rfma(A3, Fz, rmul(orh45, uz));
  const Real gmag = radd(sqrt(rfma(gzv, gzv, rfma(gyv, gyv, rmul(gxv, gxv)))), (Real)1e-12);
  const Real sh = rmul(rmul(sharpC4, p), rsub(one, p)) / gmag;
  const Real D0 = rmul(omP, p);
  const Real fp = rmul((Real)4, D0);
  const Real Dx = rfma(sh, gxv, rmul(fp, ux)), Dy = rfma(sh, gyv, rmul(fp, uy)), Dz = rfma(sh, gzv, rmul(fp, uz));
  const Real om1 = rsub(one, om), omP1 = rsub(one, omP);
  static_for<0, Q27>([&](auto KK) {
    constexpr int k = decltype(KK)::value;
    using D = D27<k>;
    constexpr int ex = D::ex, ey = D::ey, ez = D::ez;
    if constexpr (MODE != 1 || halo_dir<SX, SY, k>()) {
      const Real ev = edot<ex, ey, ez>(Vx, Vy, Vz);
      const Real eu = edot<ex, ey, ez>(ux, uy, uz);
      const Real eq = edot<ex, ey, ez>(Qx, Qy, Qz);
      const Real w = (Real)D::w;
      // f*_k = (1 - w) f_k + (w_k T + w_k e.V) with T = (e.u)(e.Q) + C0.  The
      // opposite direction has the same T and the negated w_k e.V, exactly
      // (every negation is exact), so a tile cell evaluates opposite pairs
      // (k odd, k + 1) together and still gets, bit for bit, what a halo
      // cell evaluating one direction alone gets.
      if constexpr (MODE == 0 && k > 0) {
        if constexpr (k & 1) {
          const Real T = rfma(eu, eq, C0), wev = rmul(w, ev), wT = rmul(w, T);
          o.f[k] = rfma(om1, C::dec(L.fv[k], w), radd(wT, wev));
          o.f[D::opp] = rfma(om1, C::dec(L.fv[D::opp], w), rsub(wT, wev));
        }
      } else {
        const Real T = rfma(eu, eq, C0), wev = rmul(w, ev), wT = rmul(w, T);
        o.f[k] = rfma(om1, C::dec(L.fv[k], w), radd(wT, wev));
      }
      if constexpr (k < Q7) {
        const Real w7 = (Real)D7<k>::w;
        // D3Q7 directions have at most one non-zero component
        const Real ed = edot<ex, ey, ez>(Dx, Dy, Dz);
        Real href = 0;
        if constexpr (C::offset) href = rmul(w7, p);
        o.h[k] = rfma(omP1, C::dec(L.hv[k], href), rmul(w7, k == 0 ? D0 : radd(D0, ed)));
      }
    }
  });
  ogx = gxv;
  ogy = gyv;
  ogz = gzv;
  olap = lap;
  ophi = p;
}

// One tile (bx, by) of 32 x TY columns over z-chunk bz of one scene.
// WIDE: 64-bit population offsets, for grids whose populations exceed 2^31
// elements (more than ~76 M cells); 32-bit offsets otherwise.
template <class PopT, int TY, bool WIDE, bool PACK = false>
__device__ __forceinline__ void fused_tile(const FusedArgs<PopT> &a, int bx, int by, int bz) {
  using POff = std::conditional_t<WIDE, long long, int>;
  using Real = typename Prec<PopT>::Real;
  using C = Codec<PopT>;
  using SM = FusedSmem<PopT, TY>;
  using LD = CellLoad<PopT>;
  using CO = CellOut<PopT>;
  constexpr int RX = SM::RX, NC = SM::NC;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Real *ring = reinterpret_cast<Real *>(smem_raw);                        // [78][NC]
  uint8_t *stag = smem_raw + SM::ringBytes;                               // [3][NC]

  const auto &s = a.s;
  const SolidSet &ss = *a.ss;
  const int cur = a.cur, nxt = 1 - cur;
  const PopT *__restrict__ Fc = s.F[cur];
  const PopT *__restrict__ Hc = s.H[cur];
  PopT *__restrict__ Fn = s.F[nxt];
  PopT *__restrict__ Hn = s.H[nxt];
  const Real *__restrict__ phiC = s.phi[cur];
  const Real *__restrict__ rhoC = s.rho[cur];
  const Real *__restrict__ uxC = s.ux[cur];
  const Real *__restrict__ uyC = s.uy[cur];
  // ux, uy in the pad slots of f's and h's last groups (FP32 / FP64 storage)
  constexpr bool UPAD = Scene<PopT, Real>::UPAD;
  const Real *__restrict__ uzC = s.uz[cur];
  const uint8_t *__restrict__ tagA = s.tag;
  const int nx = s.nx, ny = s.ny, nz = s.nz, nxny = nx * ny;
  const long long nCell = s.n, nF = pop_elems(s.n, Q27), nH = pop_elems(s.n, Q7);
  constexpr int RING = RING_PLANES * NC, TAGS = 3 * NC;
  constexpr int G27 = PopGroups<Q27>::G, G7 = PopGroups<Q7>::G;
  constexpr int BLK27 = PopGroups<Q27>::BLOCK, BLK7 = PopGroups<Q7>::BLOCK;
  const Real om = (Real)a.om, omP = (Real)a.omP, A = (Real)a.A;
  const Real beta4 = (Real)a.beta4, kappa = (Real)a.kappa, rhoG = (Real)a.rhoG;
  const Real dRho = (Real)a.dRho, grav = (Real)a.gravity, sharpC4 = (Real)a.sharpC4;

  const int tx = threadIdx.x, ty = threadIdx.y;
  const bool haloA = ty == TY, haloWarp = ty >= TY;
  const int x0 = bx * 32, y0 = by * TY;
  const int zb = 1 + bz * a.zchunk;
  const int ze = min(zb + a.zchunk, nz - 1);
  if (zb >= ze) return;
  const int x = x0 + tx, y = y0 + ty;
  const int own = (ty + 1) * RX + (tx + 1);

  // Side lane of halo warp B: 0..TY-1 left column, TY..2TY-1 right column,
  // then the four corners (0,0) (33,0) (0,TY+1) (33,TY+1); others idle.
  int sideLx = 0, sideLy = 0, sideSx = 2, sideSy = 2;
  const bool sideAct = tx < 2 * TY + 4;
  if (tx < TY) {
    sideLx = 0, sideLy = tx + 1, sideSx = 1, sideSy = 0;
  } else if (tx < 2 * TY) {
    sideLx = RX - 1, sideLy = tx - TY + 1, sideSx = -1, sideSy = 0;
  } else if (sideAct) {
    const int c = tx - 2 * TY;
    sideLx = (c & 1) ? RX - 1 : 0;
    sideLy = (c & 2) ? TY + 1 : 0;
    sideSx = (c & 1) ? -1 : 1;
    sideSy = (c & 2) ? -1 : 1;
  }

  // Directions a pass needs: MODE 0 all (a tile cell); MODE 1 the compile-time
  // halo side (SX, SY); MODE 2 the run-time side (sx, sy), none when inactive.
  auto needs = [&](auto MODEc, auto SXc, auto SYc, auto KK, int sx, int sy,
                   bool active) __attribute__((always_inline)) -> bool {
    constexpr int MODE = decltype(MODEc)::value, SX = decltype(SXc)::value, SY = decltype(SYc)::value;
    constexpr int k = decltype(KK)::value;
    if constexpr (MODE == 0) return true;
    else if constexpr (MODE == 1) return halo_dir<SX, SY, k>();
    else return active && (sx == 0 || D27<k>::ex == sx) && (sy == 0 || D27<k>::ey == sy);
  };

  // Load phase: every load comes from a valid, clamped address and none waits
  // on the tag, so a pass costs one memory latency.
  // The phi stencil, rho, u and tag of cell (gx_, gy_, q).
  auto load_small = [&](int q, int gx_, int gy_, LD &L) __attribute__((always_inline)) {
    const bool inside = gx_ >= 0 && gx_ < nx && gy_ >= 0 && gy_ < ny && q >= 0 && q < nz;
    const int ci = inside ? q * nxny + gy_ * nx + gx_ : 0;
    uint8_t tg = ldg_at(tagA, ci, nCell, 1);
    const int last = (int)nCell - 1;
    L.p = ldg_at(phiC, ci, nCell, 5);
    L.pxp = ldg_at(phiC, min(ci + 1, last), nCell, 5);
    L.pxm = ldg_at(phiC, max(ci - 1, 0), nCell, 5);
    L.pyp = ldg_at(phiC, min(ci + nx, last), nCell, 5);
    L.pym = ldg_at(phiC, max(ci - nx, 0), nCell, 5);
    L.pzp = ldg_at(phiC, min(ci + nxny, last), nCell, 5);
    L.pzm = ldg_at(phiC, max(ci - nxny, 0), nCell, 5);
    L.sumF = ldg_at(rhoC, ci, nCell, 6);
    if constexpr (UPAD) {
      L.ux = (Real)ldg_at(Fc, (long long)(ci >> 3) * BLK27 + (ci & 7) * 4 + pofs(27), nF, 6);
      L.uy = (Real)ldg_at(Hc, (long long)(ci >> 3) * BLK7 + (ci & 7) * 4 + pofs(7), nH, 6);
    } else {
      L.ux = ldg_at(uxC, ci, nCell, 6);
      L.uy = ldg_at(uyC, ci, nCell, 6);
    }
    L.uz = ldg_at(uzC, ci, nCell, 6);
    // boundary cells never act as fluid (they are walls after any retag)
    const bool inner = gx_ >= 1 && gx_ <= nx - 2 && gy_ >= 1 && gy_ <= ny - 2 && q >= 1 && q <= nz - 2;
    if (!inside || (!inner && tg == TAG_FLUID)) tg = TAG_WALL;
    L.tg = tg;
  };
  auto load = [&](auto MODEc, auto SXc, auto SYc, int sx, int sy, bool active, int q, int gx_, int gy_,
                  LD &L) __attribute__((always_inline)) {
    constexpr int MODE = decltype(MODEc)::value, SX = decltype(SXc)::value, SY = decltype(SYc)::value;
    const bool inside = gx_ >= 0 && gx_ < nx && gy_ >= 0 && gy_ < ny && q >= 0 && q < nz;
    const int ci = inside ? q * nxny + gy_ * nx + gx_ : 0;
    const POff bF = (POff)(ci >> 3) * BLK27 + (ci & 7) * 4;
    const POff bH = (POff)(ci >> 3) * BLK7 + (ci & 7) * 4;
    // whole groups of four directions, loaded when any of their directions is needed
    auto groups = [&](auto QQ, auto NG, const PopT *src, POff base, long long lim, int code,
                      PopT *dst) __attribute__((always_inline)) {
      constexpr int Q = decltype(QQ)::value;
      static_for<0, decltype(NG)::value>([&](auto GG) {
        constexpr int g = decltype(GG)::value;
        if constexpr (MODE != 1 || halo_group<SX, SY, Q, g>()) {
          bool nd = false;
          static_for<4 * g, (4 * g + 4 < Q ? 4 * g + 4 : Q)>([&](auto KK) {
            nd = nd || needs(MODEc, SXc, SYc, KK, sx, sy, active);
          });
          PopT t[4];
          ldg4_at(src, base + 32 * g, lim, code, nd, t);
          static_for<4 * g, (4 * g + 4 < Q ? 4 * g + 4 : Q)>([&](auto KK) {
            constexpr int k = decltype(KK)::value;
            dst[k] = t[k & 3];
          });
        }
      });
    };
    groups(IC<Q27>{}, IC<G27>{}, Fc, bF, nF, 3, L.fv);
    groups(IC<Q7>{}, IC<G7>{}, Hc, bH, nH, 4, L.hv);
    load_small(q, gx_, gy_, L);
  };

  // Emit phase: the collided values and the tag of a cell into ring cell lc of
  // plane q.  Values computed for non-fluid cells land in ring slots that are
  // never read as sources.
  auto emit = [&](auto MODEc, auto SXc, auto SYc, int sx, int sy, bool active, int q, int lc,
                  const CO &o) __attribute__((always_inline)) {
    constexpr int MODE = decltype(MODEc)::value, SX = decltype(SXc)::value, SY = decltype(SYc)::value;
    const int fbM = (RING_F_M + (q & 1) * 9) * NC + lc, fbZ = (RING_F_Z + (q & 1) * 9) * NC + lc;
    const int fbP = (RING_F_P + (q % 3) * 9) * NC + lc;
    const int hbM = (RING_H_M + (q & 1)) * NC + lc, hbZ = (RING_H_Z + (q & 1) * 5) * NC + lc;
    const int hbP = (RING_H_P + (q % 3)) * NC + lc;
    if (MODE != 2 || active) stag[sm_at((q % 3) * NC + lc, TAGS, 2)] = (MODE == 1 && SY < 0) ? o.tg2 : o.tg;
    static_for<0, Q27>([&](auto KK) {
      constexpr int k = decltype(KK)::value;
      using D = D27<k>;
      constexpr int ez = D::ez;
      if constexpr (MODE != 1 || halo_dir<SX, SY, k>()) {
        const bool nd = needs(MODEc, SXc, SYc, KK, sx, sy, active);
        const int fb = ez < 0 ? fbM : (ez == 0 ? fbZ : fbP);
        if (nd) ring[sm_at(fb + slot27(k) * NC, RING, 7)] = o.f[k];
        if constexpr (k < Q7) {
          const int hb = ez < 0 ? hbM : (ez == 0 ? hbZ : hbP);
          if (nd) ring[sm_at(hb + (ez == 0 ? k : 0) * NC, RING, 8)] = o.h[k];
        }
      }
    });
  };

  // Compute phase: the collision of one cell into registers (o), for emit.
  const CollK<Real> K = coll_consts(a);
  auto compute = [&](auto MODEc, auto SXc, auto SYc, const LD &L, CO &o, Real &ogx, Real &ogy, Real &ogz, Real &olap,
                     Real &ophi) __attribute__((always_inline)) {
    collide_cell<PopT, decltype(MODEc)::value, decltype(SXc)::value, decltype(SYc)::value>(K, L, o, ogx, ogy, ogz,
                                                                                         olap, ophi);
  };

  // Collide plane q: cell warps their own cells; halo warp A the rows above
  // and below the tile (both rows loaded before either is computed); halo
  // warp B the side columns and corners.
  // (lambdas are forced inline: an outlined closure would live in local memory)
  auto halo_plane = [&](int q, CO &o) __attribute__((always_inline)) {
    Real d0, d1, d2, d3, d4;
    if (haloA) {
      LD top, bot;
      load(IC<1>{}, IC<0>{}, IC<1>{}, 0, 0, true, q, x, y0 - 1, top);
      load(IC<1>{}, IC<0>{}, IC<-1>{}, 0, 0, true, q, x, y0 + TY, bot);
      compute(IC<1>{}, IC<0>{}, IC<1>{}, top, o, d0, d1, d2, d3, d4);
      compute(IC<1>{}, IC<0>{}, IC<-1>{}, bot, o, d0, d1, d2, d3, d4);
    } else {
      LD L;
      load(IC<2>{}, IC<0>{}, IC<0>{}, sideSx, sideSy, sideAct, q, x0 - 1 + sideLx, y0 - 1 + sideLy, L);
      compute(IC<2>{}, IC<0>{}, IC<0>{}, L, o, d0, d1, d2, d3, d4);
    }
  };
  // collide plane q into registers (o: a cell warp's cell, halo warp A's two
  // rows, halo warp B's side cell) ...
  auto collide_plane = [&](int q, CO &o, Real &ogx, Real &ogy, Real &ogz, Real &olap,
                           Real &ophi) __attribute__((always_inline)) {
    if (!haloWarp) {
      LD L;
      load(IC<0>{}, IC<0>{}, IC<0>{}, 0, 0, true, q, x, y, L);
      compute(IC<0>{}, IC<0>{}, IC<0>{}, L, o, ogx, ogy, ogz, olap, ophi);
    } else {
      halo_plane(q, o);
    }
  };
  // ... and from registers into the ring
  auto emit_plane = [&](int q, const CO &o) __attribute__((always_inline)) {
    if (!haloWarp) {
      emit(IC<0>{}, IC<0>{}, IC<0>{}, 0, 0, true, q, own, o);
    } else if (haloA) {
      emit(IC<1>{}, IC<0>{}, IC<1>{}, 0, 0, true, q, tx + 1, o);
      emit(IC<1>{}, IC<0>{}, IC<-1>{}, 0, 0, true, q, (TY + 1) * RX + tx + 1, o);
    } else {
      emit(IC<2>{}, IC<0>{}, IC<0>{}, sideSx, sideSy, sideAct, q, sideLy * RX + sideLx, o);
    }
  };

  Real gxC = 0, gyC = 0, gzC = 0, lapC = 0, phC = 0;
  Real gxN = 0, gyN = 0, gzN = 0, lapN = 0, phN = 0;
  const bool colActive = !haloWarp && x >= 1 && x <= nx - 2 && y >= 1 && y <= ny - 2;

  // Iteration q collides plane q and pulls plane q - 1 (planes zb-1 .. ze are
  // collided, zb .. ze-1 pulled): load and collide plane q into registers,
  // barrier (every warp has pulled plane q - 2), write the ring, barrier, pull
  // plane q - 1.
  for (int q = zb - 1; q <= ze; q++) {
    CO o;
    collide_plane(q, o, gxN, gyN, gzN, lapN, phN);
    // plane q's slots of the ring are free once every warp has pulled plane
    // q - 2; a warp that gets here early has its loads and collision of plane
    // q behind it
    __syncthreads();
    emit_plane(q, o);
    __syncthreads();
    // pull plane z = q - 1 (nothing while z < zb)
    const int z = q - 1;
    const int sC = (z + 3) % 3;
    const uint8_t tagI = colActive && z >= zb ? stag[sm_at(sC * NC + own, TAGS, 9)] : TAG_WALL;
    const int i = z * nxny + y * nx + x;
    const POff bF = (POff)(i >> 3) * BLK27 + (i & 7) * 4;
    const POff bH = (POff)(i >> 3) * BLK7 + (i & 7) * 4;
    if (tagI == TAG_SOLID) {
      // Solid cells are not updated; carry their state into the next half so
      // both halves hold the reference's stale values.
#pragma unroll 1
      for (int g = 0; g < G27; g++) {
        PopT t[4];
        ldg4_at(Fc, bF + 32 * g, nF, 10, true, t);
        st4_at(Fn, bF + 32 * g, nF, 10, t);
      }
#pragma unroll 1
      for (int g = 0; g < G7; g++) {
        PopT t[4];
        ldg4_at(Hc, bH + 32 * g, nH, 11, true, t);
        st4_at(Hn, bH + 32 * g, nH, 11, t);
      }
      st_at(s.phi[nxt], i, nCell, 12, ldg_at(phiC, i, nCell, 12));
      st_at(s.rho[nxt], i, nCell, 12, ldg_at(rhoC, i, nCell, 12));
      if constexpr (!UPAD) {  // (in the pads, copied with the groups above)
        st_at(s.ux[nxt], i, nCell, 12, ldg_at(uxC, i, nCell, 12));
        st_at(s.uy[nxt], i, nCell, 12, ldg_at(uyC, i, nCell, 12));
      }
      st_at(s.uz[nxt], i, nCell, 12, ldg_at(uzC, i, nCell, 12));
      if (PACK && lbm_ok(i < nCell, 50, i)) pack_rg8(a.pack, i, ldg_at(phiC, i, nCell, 12), true);
    } else if (tagI == TAG_FLUID) {
      // ring bases: group e_z sources come from plane z - e_z; the cell's own
      // (bounce-back) values are in plane z
      const int sbFM = (RING_F_M + ((z + 1) & 1) * 9) * NC + own;
      const int sbFZ = (RING_F_Z + (z & 1) * 9) * NC + own;
      const int sbFP = (RING_F_P + ((z + 2) % 3) * 9) * NC + own;
      const int obFM = (RING_F_M + (z & 1) * 9) * NC + own;
      const int obFP = (RING_F_P + (z % 3) * 9) * NC + own;
      const int sbHM = (RING_H_M + ((z + 1) & 1)) * NC + own;
      const int sbHZ = (RING_H_Z + (z & 1) * 5) * NC + own;
      const int sbHP = (RING_H_P + ((z + 2) % 3)) * NC + own;
      const int obHM = (RING_H_M + (z & 1)) * NC + own;
      const int obHP = (RING_H_P + (z % 3)) * NC + own;
      const int tbM = ((z + 1) % 3) * NC + own, tbZ = sC * NC + own, tbP = ((z + 2) % 3) * NC + own;
      const Real rhoPhOld = rfma(phC, dRho, rhoG);
      Real rhoA = 0, mx = 0, my = 0, mz = 0, hsum = 0;
      Real hn[Q7];
      Real val4[4], ref4[4];  // the current group's values and offsets, encoded and stored as one vector
      PopT enc4[4];
      uint32_t orTags = 0;  // OR of the source tags: bit TAG_SOLID set iff a source is SOLID
      static_for<0, Q27>([&](auto KK) {
        constexpr int k = decltype(KK)::value;
        using D = D27<k>;
        constexpr int ex = D::ex, ey = D::ey, ez = D::ez, o = D::opp;
        constexpr int oz = D27<o>::ez;
        constexpr int so = -ey * RX - ex;  // source offset in the ring plane
        const int tb = ez < 0 ? tbM : (ez == 0 ? tbZ : tbP);
        const int sbF = ez < 0 ? sbFM : (ez == 0 ? sbFZ : sbFP);
        const int obF = oz < 0 ? obFM : (oz == 0 ? sbFZ : obFP);
        const uint8_t ts = stag[sm_at(tb + so, TAGS, 13)];
        const bool fl = ts == TAG_FLUID;
        // fluid source: its post-collision value; otherwise halfway bounce-back
        // of the cell's own opposite value (moving-wall term added below).
        // Both slots are read and the value selected, so each load keeps its
        // compile-time offset and no address is selected per direction.
#ifdef LBM_CHECKED
        const Real fk = ring[sm_at(fl ? sbF + slot27(k) * NC + so : obF + slot27(o) * NC, RING, 14)];
#else
        const Real fS = ring[sbF + slot27(k) * NC + so];
        const Real fO = ring[obF + slot27(o) * NC];
        const Real fk = fl ? fS : fO;
#endif
        orTags |= ts;
        val4[k & 3] = fk;
        ref4[k & 3] = (Real)D::w;
        if constexpr ((k & 3) == 3 || k == Q27 - 1) {
          if constexpr (k == Q27 - 1) val4[3] = ref4[3] = 0;  // pad of the last group: encodes to +0
          C::enc4(val4, ref4, enc4);
          st4_at(Fn, bF + pofs(k & ~3), nF, 15, enc4);
        }
        rhoA += fk;
        if constexpr (ex != 0) mx += (Real)ex * fk;
        if constexpr (ey != 0) my += (Real)ey * fk;
        if constexpr (ez != 0) mz += (Real)ez * fk;
        if constexpr (k < Q7) {
          constexpr int hs = (ez == 0 ? k : 0), hso = (oz == 0 ? o : 0);
          const int sbH = ez < 0 ? sbHM : (ez == 0 ? sbHZ : sbHP);
          const int obH = oz < 0 ? obHM : (oz == 0 ? sbHZ : obHP);
#ifdef LBM_CHECKED
          const Real hk = ring[sm_at(fl ? sbH + hs * NC + so : obH + hso * NC, RING, 16)];
#else
          const Real hS = ring[sbH + hs * NC + so];
          const Real hO = ring[obH + hso * NC];
          const Real hk = fl ? hS : hO;
#endif
          hn[k] = hk;
          hsum += hk;
        }
      });
      // Links to SOLID sources (rare): Ladd moving-wall term
      // 2 w_k rho_phase(phi_old) (e_k . u_s) / cs^2 and the FP64 momentum
      // exchange -(f_opp + f_k) e_k at the solid cell (src/sim.js:517-536).
      static_assert(TAG_FLUID == 0 && (TAG_SOLID & TAG_WALL) == 0, "tag bits");
      if (orTags & TAG_SOLID) {
        uint32_t solidM = 0;
#pragma unroll 1
        for (int k = 1; k < Q27; k++) {
          const int ez = dcomp(k, 2);
          const int tb = ez < 0 ? tbM : (ez == 0 ? tbZ : tbP);
          const int so = -dcomp(k, 1) * RX - dcomp(k, 0);
          if (stag[sm_at(tb + so, TAGS, 13)] == TAG_SOLID) solidM |= 1u << k;
        }
        double acc[6] = {0, 0, 0, 0, 0, 0};
        int owner = -1;
        for (uint32_t m = solidM; m; m &= m - 1) {
          const int k = __ffs(m) - 1;
          const int ex = dcomp(k, 0), ey = dcomp(k, 1), ez = dcomp(k, 2);
          const int o = opp_of(k), oz = -ez;
          const int sx = x - ex, sy = y - ey, sz = z - ez;
          const int b = owner_of<LBM_MAX_SPHERES>(ss.sph, ss.nsph, sx, sy, sz);
          if (b < 0) continue;
          double ox, oy, oz_;
          sphere_surface_velocity(ss.sph[b], sx, sy, sz, ox, oy, oz_);
          // surface velocity rounded as the reference stores it (Float32Array us)
          const Real eus = (Real)ex * (Real)ox + (Real)ey * (Real)oy + (Real)ez * (Real)oz_;
          const Real w = (Real)w27_of(k);
          const Real corr = (Real)2 * w * rhoPhOld * eus * (Real)3;
          const int obF = oz < 0 ? obFM : (oz == 0 ? sbFZ : obFP);
          const Real fopp = ring[sm_at(obF + c_slot27[o] * NC, RING, 19)];
          const Real fk = fopp + corr;
          st_at(Fn, bF + pofs(k), nF, 15, C::enc(fk, w));
          rhoA += corr;
          mx += (Real)ex * corr;
          my += (Real)ey * corr;
          mz += (Real)ez * corr;
          if (b != owner) {
            flush_impulse(ss, owner, x, y, z, acc);
            owner = b;
          }
          const double mom = __dadd_rn((double)fopp, (double)fk);
          impulse_terms(ss.sph[b], sx, sy, sz, -mom * ex, -mom * ey, -mom * ez, acc);
        }
        flush_impulse(ss, owner, x, y, z, acc);
      }

      // macros (src/sim.js:545-576)
      const Real rhoN = rhoA > (Real)0.01 ? rhoA : (Real)0.01;
      const Real p = hsum < (Real)0 ? (Real)0 : hsum > (Real)1 ? (Real)1 : hsum;
      static_for<0, Q7>([&](auto KK) {
        constexpr int k = decltype(KK)::value;
        val4[k & 3] = hn[k];
        ref4[k & 3] = (Real)D7<k>::w * p;
        if constexpr ((k & 3) == 3 || k == Q7 - 1) {
          if constexpr (k == Q7 - 1) val4[3] = ref4[3] = 0;
          C::enc4(val4, ref4, enc4);
          st4_at(Hn, bH + pofs(k & ~3), nH, 17, enc4);
        }
      });
      // explicitly rounded like the collision, so every instance of this
      // kernel (tile shapes, staged or not, batched or not) gives the same bits
      const Real one = (Real)1, half = (Real)0.5;
      const Real rhoPhN = rfma(p, dRho, rhoG);
      const Real mu = rfma(-kappa, lapC, rmul(rmul(rmul(beta4, p), rsub(p, one)), rfma((Real)2, p, -one)));
      const Real Fx = rmul(mu, gxC), Fy = rfma(mu, gyC, rmul(rhoPhN, grav)), Fz = rmul(mu, gzC);
      const Real inv = one / rhoPhN;
      Real uxn = rmul(rfma(half, Fx, mx), inv);
      Real uyn = rmul(rfma(half, Fy, my), inv);
      Real uzn = rmul(rfma(half, Fz, mz), inv);
      const Real u2 = rfma(uzn, uzn, rfma(uyn, uyn, rmul(uxn, uxn)));
      if (u2 > (Real)(0.2 * 0.2)) {
        const Real sc = (Real)0.2 / sqrt(u2);
        uxn = rmul(uxn, sc);
        uyn = rmul(uyn, sc);
        uzn = rmul(uzn, sc);
      }
      st_at(s.rho[nxt], i, nCell, 18, rhoN);
      st_at(s.phi[nxt], i, nCell, 18, p);
      if constexpr (UPAD) {
        // into the pads of the groups stored above (the same sectors)
        st_at(Fn, bF + pofs(27), nF, 18, (PopT)uxn);
        st_at(Hn, bH + pofs(7), nH, 18, (PopT)uyn);
      } else {
        st_at(s.ux[nxt], i, nCell, 18, uxn);
        st_at(s.uy[nxt], i, nCell, 18, uyn);
      }
      st_at(s.uz[nxt], i, nCell, 18, uzn);
      if (PACK && lbm_ok(i < nCell, 50, i)) pack_rg8(a.pack, i, p, false);
    } else if (PACK && !haloWarp && x < nx && y < ny && z >= zb) {
      // a wall cell of this tile: not updated, packed from the half that is
      // current after the step
      if (lbm_ok(i < nCell, 50, i)) pack_rg8(a.pack, i, ldg_at(s.phi[nxt], i, nCell, 12), false);
    }
    gxC = gxN;
    gyC = gyN;
    gzC = gzN;
    lapC = lapN;
    phC = phN;
  }
}

// One scene: the grid is its tiles.
// PACK: the instance launched on frame steps, which also writes the RG8
// volume; the other steps run an instance without that code
template <class PopT, int TY, bool WIDE, bool PACK = false>
__global__ void __launch_bounds__(32 * (TY + 2), FusedOcc<PopT, TY>::blocks)
    k_fused_step(const __grid_constant__ FusedArgs<PopT> a) {
  fused_tile<PopT, TY, WIDE, PACK>(a, blockIdx.x, blockIdx.y, blockIdx.z);
}

// Many scenes in one persistent launch: tile w of the batch belongs to the
// scene s with tileStart[s] <= w < tileStart[s+1]; each scene's descriptor
// gives its own grid, physics constants and state.  CTAs stride over the
// tiles, so one launch of about one wave advances every scene by a step.
template <class PopT, int TY, bool WIDE>
__global__ void __launch_bounds__(32 * (TY + 2), FusedOcc<PopT, TY>::blocks)
    k_fused_batch(const FusedArgs<PopT> *__restrict__ args, const int *__restrict__ tileStart,
                  const int3 *__restrict__ tileGrid, int nscenes) {
  const int total = tileStart[nscenes];
  for (int w = blockIdx.x; w < total; w += gridDim.x) {
    int lo = 0, hi = nscenes - 1;  // last scene whose first tile is <= w
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (tileStart[mid] <= w) lo = mid;
      else hi = mid - 1;
    }
    const int3 g = tileGrid[lo];
    const int t = w - tileStart[lo];
    const int bx = t % g.x, by = (t / g.x) % g.y, bz = t / (g.x * g.y);
    // the scene's descriptor in shared memory: its fields are re-read there
    // instead of being held in registers through the tile
    __shared__ FusedArgs<PopT> sa;
    constexpr int WORDS = sizeof(FusedArgs<PopT>) / 4;
    static_assert(sizeof(FusedArgs<PopT>) % 4 == 0, "descriptor copied in words");
    const int lin = threadIdx.y * blockDim.x + threadIdx.x;
    if (lin < WORDS)
      reinterpret_cast<uint32_t *>(&sa)[lin] = reinterpret_cast<const uint32_t *>(args + lo)[lin];
    __syncthreads();
    fused_tile<PopT, TY, WIDE>(sa, bx, by, bz);
    __syncthreads();  // the next tile reuses shared memory
  }
}

}  // namespace lbm
