// Kernel templates of the LBM step.  Included by one translation unit per
// population storage type (lbm_inst_*.cu), which instantiates Ops<PopT>.
//
// Two execution forms share one device state:
//  * phase-by-phase kernels that mirror the reference's seven Sim methods one
//    to one (src/sim.js:176-582), for callers that invoke them individually;
//  * the fused step: a z-marching kernel that, per cell, pulls the 27 + 7
//    populations of its neighbours, applies each source cell's BGK collision on
//    the fly from per-cell collision coefficients staged in shared memory,
//    streams with halfway bounce-back / moving-wall correction, and writes the
//    new populations and macros -- one read and one write of every state array
//    per step.
#pragma once

#include <stdio.h>

#include "lbm_core.cuh"

namespace lbm {

template <class PopT>
struct Prec {
  using Real = float;
};
template <>
struct Prec<double> {
  using Real = double;
};

inline unsigned nblocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

__device__ __forceinline__ long long cell_index(int x, int y, int z, int nx, int ny) {
  return ((long long)z * ny + y) * nx + x;
}

// The reference's phase loops run over 1..n-2 on every axis (src/sim.js:334-338);
// cells on the boundary are never collided or streamed, whatever their tag.
__device__ __forceinline__ bool interior_cell(long long i, int nx, int ny, int nz) {
  int x = (int)(i % nx);
  long long t = i / nx;
  int y = (int)(t % ny);
  int z = (int)(t / ny);
  return x >= 1 && x <= nx - 2 && y >= 1 && y <= ny - 2 && z >= 1 && z <= nz - 2;
}

// Weight tables usable with a runtime index (generic kernels, host code).
__host__ __device__ inline float w27_of(int k) {
  int nnz = (dcomp(k, 0) != 0) + (dcomp(k, 1) != 0) + (dcomp(k, 2) != 0);
  return (float)(nnz == 0 ? 8.0 / 27.0 : nnz == 1 ? 2.0 / 27.0 : nnz == 2 ? 1.0 / 54.0 : 1.0 / 216.0);
}
__host__ __device__ inline float w7_of(int k) { return (float)(k == 0 ? 0.25 : 0.125); }
__host__ __device__ inline int opp_of(int k) { return k == 0 ? 0 : ((k & 1) ? k + 1 : k - 1); }

__device__ __forceinline__ void flush_impulse(const SolidSet &ss, int owner, int x, int y, int z,
                                              double acc[6]) {
  if (owner < 0) return;
  const ImpulseTarget &t = ss.imp[owner];
  int lx = x - t.lo[0], ly = y - t.lo[1], lz = z - t.lo[2];
  if (lx < 0 || ly < 0 || lz < 0 || lx >= t.dim[0] || ly >= t.dim[1] || lz >= t.dim[2]) return;
  double *slot = t.acc + 6 * (((long long)lz * t.dim[1] + ly) * t.dim[0] + lx);
#pragma unroll
  for (int j = 0; j < 6; j++) {
    slot[j] = __dadd_rn(slot[j], acc[j]);
    acc[j] = 0.0;
  }
}

// =====================================================================================
// init (src/sim.js:112-134): both ping-pong halves receive identical values so
// that walls, which are never rewritten, read the same from either half.
template <class PopT>
__global__ void k_init_flat(Scene<PopT, typename Prec<PopT>::Real> s, const double *phiCol) {
  using Real = typename Prec<PopT>::Real;
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= s.n) return;
  int x = (int)(i % s.nx);
  long long t = i / s.nx;
  int y = (int)(t % s.ny);
  int z = (int)(t / s.ny);
  double pc = phiCol[y];
  bool wall = x == 0 || x == s.nx - 1 || y == 0 || y == s.ny - 1 || z == 0 || z == s.nz - 1;
  Real phiR = (Real)pc;
  for (int c = 0; c < 2; c++) {
    s.phi[c][i] = phiR;
    s.rho[c][i] = (Real)1.0;
    s.set_ux(c, i, (Real)0);
    s.set_uy(c, i, (Real)0);
    s.uz[c][i] = (Real)0;
    for (int k = 0; k < Q27; k++) {
      Real w = (Real)w27_of(k);
      s.F[c][pidx<27>(k, i)] = Codec<PopT>::enc(w, w);
    }
    for (int k = 0; k < Q7; k++) {
      Real hv = (Real)((double)w7_of(k) * pc);
      s.H[c][pidx<7>(k, i)] = Codec<PopT>::enc(hv, (Real)w7_of(k) * phiR);
    }
  }
  uint8_t tg = wall ? TAG_WALL : TAG_FLUID;
  s.tag[i] = tg;
  s.tagPrev[i] = tg;
}

// seedHydrostatic (src/sim.js:144-173): one thread per (z, x) column, y
// ascending, FP64 arithmetic; writes rho and f into both halves.
template <class PopT>
__global__ void k_seed_hydrostatic(Scene<PopT, typename Prec<PopT>::Real> s, int cur, double rhoL,
                                   double rhoG, double gravity) {
  using Real = typename Prec<PopT>::Real;
  long long col = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (col >= (long long)s.nx * s.nz) return;
  int x = (int)(col % s.nx);
  int z = (int)(col / s.nx);
  const double dRho = rhoL - rhoG;
  const double gOverCs2 = gravity * 3.0;
  const double uLatY = -0.5 * gravity;
  const double uLat2 = uLatY * uLatY;
  double pCs2 = 1.0;
  for (int y = 0; y < s.ny; y++) {
    long long i = cell_index(x, y, z, s.nx, s.ny);
    double rhoPhase = rhoG + (double)s.phi[cur][i] * dRho;
    for (int c = 0; c < 2; c++) s.rho[c][i] = (Real)pCs2;
    for (int k = 0; k < Q27; k++) {
      double eu = dcomp(k, 1) * uLatY;
      double Qi = eu * (3.0 + 4.5 * eu) - 1.5 * uLat2;
      double fk = (double)w27_of(k) * (pCs2 + rhoPhase * Qi);
      Real w = (Real)w27_of(k);
      PopT e = Codec<PopT>::enc((Real)fk, w);
      s.F[0][pidx<27>(k, i)] = e;
      s.F[1][pidx<27>(k, i)] = e;
    }
    pCs2 += rhoPhase * gOverCs2;
  }
}

// =====================================================================================
// Phase-by-phase kernels (FP32 and FP64 storage).  Reference semantics:
// f = F[cur], f2 = F[1-cur]; h = H[cur], h2 = H[1-cur]; macros in place in
// [cur]; phiPrev = phi[1-cur].

// computePhiGradients (src/sim.js:176-199)
template <class PopT>
__global__ void k_gradients(Scene<PopT, typename Prec<PopT>::Real> s, int cur) {
  using Real = typename Prec<PopT>::Real;
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= s.n) return;
  const int nx = s.nx, ny = s.ny, nz = s.nz;
  int x = (int)(i % nx);
  long long t = i / nx;
  int y = (int)(t % ny);
  int z = (int)(t / ny);
  int zm = z > 0 ? z - 1 : z, zp = z < nz - 1 ? z + 1 : z;
  int ym = y > 0 ? y - 1 : y, yp = y < ny - 1 ? y + 1 : y;
  int xm = x > 0 ? x - 1 : x, xp = x < nx - 1 ? x + 1 : x;
  const Real *phi = s.phi[cur];
  Real c = phi[i];
  Real px = phi[cell_index(xp, y, z, nx, ny)];
  Real mx = phi[cell_index(xm, y, z, nx, ny)];
  Real py = phi[cell_index(x, yp, z, nx, ny)];
  Real my = phi[cell_index(x, ym, z, nx, ny)];
  Real pz = phi[cell_index(x, y, zp, nx, ny)];
  Real mz = phi[cell_index(x, y, zm, nx, ny)];
  s.gx[i] = (Real)0.5 * (px - mx);
  s.gy[i] = (Real)0.5 * (py - my);
  s.gz[i] = (Real)0.5 * (pz - mz);
  s.lap[i] = px + mx + py + my + pz + mz - (Real)6 * c;
}

// retagCells over the whole grid (src/sim.js:214-244): tagPrev <- tag,
// phiPrev <- phi, classification with FP64 contains, us = float(surfaceVelocity).
template <class PopT>
__global__ void k_retag_full(Scene<PopT, typename Prec<PopT>::Real> s, int cur,
                             const SolidSet *__restrict__ ssp) {
  const SolidSet &ss = *ssp;
  using Real = typename Prec<PopT>::Real;
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= s.n) return;
  const int nx = s.nx, ny = s.ny, nz = s.nz;
  int x = (int)(i % nx);
  long long t = i / nx;
  int y = (int)(t % ny);
  int z = (int)(t / ny);
  s.tagPrev[i] = s.tag[i];
  s.phi[1 - cur][i] = s.phi[cur][i];
  if (x == 0 || x == nx - 1 || y == 0 || y == ny - 1 || z == 0 || z == nz - 1) {
    s.tag[i] = TAG_WALL;
    s.usx[i] = s.usy[i] = s.usz[i] = (Real)0;
    return;
  }
  int b = owner_of<LBM_MAX_SPHERES>(ss.sph, ss.nsph, x, y, z);
  if (b >= 0) {
    double ox, oy, oz;
    sphere_surface_velocity(ss.sph[b], x, y, z, ox, oy, oz);
    s.tag[i] = TAG_SOLID;
    // stored like the reference's Float32Array us (double in the FP64 form)
    s.usx[i] = (Real)ox;
    s.usy[i] = (Real)oy;
    s.usz[i] = (Real)oz;
  } else {
    s.tag[i] = TAG_FLUID;
    s.usx[i] = s.usy[i] = s.usz[i] = (Real)0;
  }
}

// collidePhase (src/sim.js:324-364)
template <class PopT>
__global__ void k_collide_phase(Scene<PopT, typename Prec<PopT>::Real> s, int cur, StepConst k) {
  using Real = typename Prec<PopT>::Real;
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= s.n || s.tag[i] != TAG_FLUID || !interior_cell(i, s.nx, s.ny, s.nz)) return;
  const Real invTau = (Real)k.invTauPhi;
  const Real sharpC = (Real)k.sharpC;
  const Real sharpFac = (Real)4.0;
  Real p = s.phi[cur][i];
  Real uxi = s.ux_at(cur, i), uyi = s.uy_at(cur, i), uzi = s.uz[cur][i];
  Real ggx = s.gx[i], ggy = s.gy[i], ggz = s.gz[i];
  Real gmag = sqrt(ggx * ggx + ggy * ggy + ggz * ggz) + (Real)1e-12;
  Real sharpen = sharpC * p * ((Real)1 - p);
  Real Sx = sharpen * sharpFac * ggx / gmag;
  Real Sy = sharpen * sharpFac * ggy / gmag;
  Real Sz = sharpen * sharpFac * ggz / gmag;
  const PopT *h = s.H[cur];
  PopT *h2 = s.H[1 - cur];
  for (int q = 0; q < Q7; q++) {
    Real wk = (Real)w7_of(q);
    Real ex = (Real)dcomp(q, 0), ey = (Real)dcomp(q, 1), ez = (Real)dcomp(q, 2);
    Real eu = ex * uxi + ey * uyi + ez * uzi;
    Real heq = wk * p * ((Real)1 + (Real)4 * eu);
    Real Fk = wk * (ex * Sx + ey * Sy + ez * Sz);
    Real hk = Codec<PopT>::dec(h[pidx<7>(q, i)], (Real)0);
    h2[pidx<7>(q, i)] = Codec<PopT>::enc(hk - invTau * (hk - heq) + Fk, (Real)0);
  }
}

// streamPhase (src/sim.js:376-397): pull with plain bounce-back.
template <class PopT>
__global__ void k_stream_phase(Scene<PopT, typename Prec<PopT>::Real> s, int cur) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= s.n || s.tag[i] != TAG_FLUID || !interior_cell(i, s.nx, s.ny, s.nz)) return;
  const int nx = s.nx, ny = s.ny;
  const PopT *h2 = s.H[1 - cur];
  PopT *h = s.H[cur];
  for (int q = 0; q < Q7; q++) {
    long long src = i - (((long long)dcomp(q, 2) * ny + dcomp(q, 1)) * nx + dcomp(q, 0));
    h[pidx<7>(q, i)] = s.tag[src] == TAG_FLUID ? h2[pidx<7>(q, src)] : h2[pidx<7>(opp_of(q), i)];
  }
}

// collideHydro (src/sim.js:406-464)
template <class PopT>
__global__ void k_collide_hydro(Scene<PopT, typename Prec<PopT>::Real> s, int cur, StepConst k) {
  using Real = typename Prec<PopT>::Real;
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= s.n || s.tag[i] != TAG_FLUID || !interior_cell(i, s.nx, s.ny, s.nz)) return;
  const Real invTau = (Real)k.invTau;
  const Real beta = (Real)k.beta, kappa = (Real)k.kappa, dRho = (Real)k.dRho;
  const Real A = (Real)k.A, rhoG = (Real)k.rhoG, gravity = (Real)k.gravity;
  Real sumF = s.rho[cur][i];
  Real p = s.phi[cur][i];
  Real rhoPhase = rhoG + p * dRho;
  Real mu = (Real)4 * beta * p * (p - (Real)1) * ((Real)2 * p - (Real)1) - kappa * s.lap[i];
  Real bx = s.bfx ? s.bfx[i] : (Real)0, by = s.bfy ? s.bfy[i] : (Real)0, bz = s.bfz ? s.bfz[i] : (Real)0;
  Real fx = bx + mu * s.gx[i];
  Real fy = by + mu * s.gy[i] + rhoPhase * gravity;
  Real fz = bz + mu * s.gz[i];
  Real uxe = s.ux_at(cur, i), uye = s.uy_at(cur, i), uze = s.uz[cur][i];
  Real u2 = uxe * uxe + uye * uye + uze * uze;
  Real negU2half = (Real)-1.5 * u2;
  Real uF = uxe * fx + uye * fy + uze * fz;
  const PopT *f = s.F[cur];
  PopT *f2 = s.F[1 - cur];
  for (int q = 0; q < Q27; q++) {
    Real wk = (Real)w27_of(q);
    Real ex = (Real)dcomp(q, 0), ey = (Real)dcomp(q, 1), ez = (Real)dcomp(q, 2);
    Real eu = ex * uxe + ey * uye + ez * uze;
    Real Qi = negU2half + eu * ((Real)3 + (Real)4.5 * eu);
    Real feq = wk * (sumF + rhoPhase * Qi);
    Real ekF = ex * fx + ey * fy + ez * fz;
    Real Sk = A * wk * (ekF * ((Real)1 + (Real)3 * eu) - uF);
    Real fk = Codec<PopT>::dec(f[pidx<27>(q, i)], (Real)0);
    f2[pidx<27>(q, i)] = Codec<PopT>::enc(fk - invTau * (fk - feq) + Sk, (Real)0);
  }
}

// streamHydroAndMacro (src/sim.js:484-582)
template <class PopT>
__global__ void k_stream_hydro_macro(Scene<PopT, typename Prec<PopT>::Real> s, int cur,
                                     StepConst kc, const SolidSet *__restrict__ ssp) {
  const SolidSet &ss = *ssp;
  using Real = typename Prec<PopT>::Real;
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= s.n || s.tag[i] != TAG_FLUID || !interior_cell(i, s.nx, s.ny, s.nz)) return;
  const int nx = s.nx, ny = s.ny;
  int x = (int)(i % nx);
  long long t = i / nx;
  int y = (int)(t % ny);
  int z = (int)(t / ny);
  const Real beta = (Real)kc.beta, kappa = (Real)kc.kappa, dRho = (Real)kc.dRho;
  const Real rhoG = (Real)kc.rhoG, gravity = (Real)kc.gravity;
  const PopT *f2 = s.F[1 - cur];
  PopT *f = s.F[cur];
  Real rhoPhaseOld = rhoG + s.phi[cur][i] * dRho;
  Real pSumF = 0, mx = 0, my = 0, mz = 0;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  int owner = -1;
  for (int q = 0; q < Q27; q++) {
    const int ex = dcomp(q, 0), ey = dcomp(q, 1), ez = dcomp(q, 2);
    long long src = i - (((long long)ez * ny + ey) * nx + ex);
    uint8_t sTag = s.tag[src];
    Real fk;
    if (sTag == TAG_FLUID) {
      fk = Codec<PopT>::dec(f2[pidx<27>(q, src)], (Real)0);
    } else {
      Real fopp = Codec<PopT>::dec(f2[pidx<27>(opp_of(q), i)], (Real)0);
      Real corr = 0;
      if (sTag == TAG_SOLID) {
        Real eu = (Real)ex * s.usx[src] + (Real)ey * s.usy[src] + (Real)ez * s.usz[src];
        corr = (Real)2 * (Real)w27_of(q) * rhoPhaseOld * eu * (Real)3;
      }
      fk = fopp + corr;
      if (sTag == TAG_SOLID && ss.nsph > 0) {
        int sx = x - ex, sy = y - ey, sz = z - ez;
        int b = owner_of<LBM_MAX_SPHERES>(ss.sph, ss.nsph, sx, sy, sz);
        if (b >= 0) {
          if (b != owner) {
            flush_impulse(ss, owner, x, y, z, acc);
            owner = b;
          }
          double m = __dadd_rn((double)fopp, (double)fk);
          impulse_terms(ss.sph[b], sx, sy, sz, -m * ex, -m * ey, -m * ez, acc);
        }
      }
    }
    f[pidx<27>(q, i)] = Codec<PopT>::enc(fk, (Real)0);
    pSumF += fk;
    mx += (Real)ex * fk;
    my += (Real)ey * fk;
    mz += (Real)ez * fk;
  }
  flush_impulse(ss, owner, x, y, z, acc);
  s.rho[cur][i] = pSumF > (Real)0.01 ? pSumF : (Real)0.01;
  Real phiSum = 0;
  for (int q = 0; q < Q7; q++) phiSum += Codec<PopT>::dec(s.H[cur][pidx<7>(q, i)], (Real)0);
  Real p = phiSum < (Real)0 ? (Real)0 : phiSum > (Real)1 ? (Real)1 : phiSum;
  s.phi[cur][i] = p;
  Real rhoPhaseNew = rhoG + p * dRho;
  Real mu = (Real)4 * beta * p * (p - (Real)1) * ((Real)2 * p - (Real)1) - kappa * s.lap[i];
  Real bx = s.bfx ? s.bfx[i] : (Real)0, by = s.bfy ? s.bfy[i] : (Real)0, bz = s.bfz ? s.bfz[i] : (Real)0;
  Real fx = bx + mu * s.gx[i];
  Real fy = by + mu * s.gy[i] + rhoPhaseNew * gravity;
  Real fz = bz + mu * s.gz[i];
  Real invRho = (Real)1 / rhoPhaseNew;
  Real uxn = (mx + (Real)0.5 * fx) * invRho;
  Real uyn = (my + (Real)0.5 * fy) * invRho;
  Real uzn = (mz + (Real)0.5 * fz) * invRho;
  Real u2 = uxn * uxn + uyn * uyn + uzn * uzn;
  const Real UMAX = (Real)0.2, UMAX2 = (Real)(0.2 * 0.2);
  if (u2 > UMAX2) {
    Real sc = UMAX / sqrt(u2);
    uxn *= sc;
    uyn *= sc;
    uzn *= sc;
  }
  s.set_ux(cur, i, uxn);
  s.set_uy(cur, i, uyn);
  s.uz[cur][i] = uzn;
}

// =====================================================================================
// Sparse passes around the spheres.

// retag on a box (the union of the current and the two previous sphere boxes):
// every cell outside it keeps tag == tagPrev, so only the box changes.
// (the bodies of the sparse kernels take their block index and grid size, so
// that a batched launch can run them for many scenes, one grid row each)
template <class PopT>
__device__ __forceinline__ void retag_box_body(const Scene<PopT, typename Prec<PopT>::Real> &s,
                                               const Plan *__restrict__ P, unsigned bid, unsigned gdim) {
  const SolidSet &ss = P->ss;
  const Box bx = P->U;
  const int dx = bx.hi[0] - bx.lo[0] + 1, dy = bx.hi[1] - bx.lo[1] + 1, dz = bx.hi[2] - bx.lo[2] + 1;
  const long long total = (long long)dx * dy * dz;
  // grid-stride over the box the plan holds (launches are sized for the
  // largest box the step may plan, which can be far larger)
  for (long long l = bid * (long long)blockDim.x + threadIdx.x; l < total; l += (long long)gdim * blockDim.x) {
    const int x = bx.lo[0] + (int)(l % dx);
    const int y = bx.lo[1] + (int)((l / dx) % dy);
    const int z = bx.lo[2] + (int)(l / ((long long)dx * dy));
    const long long i = cell_index(x, y, z, s.nx, s.ny);
    s.tagPrev[i] = s.tag[i];
    if (x == 0 || x == s.nx - 1 || y == 0 || y == s.ny - 1 || z == 0 || z == s.nz - 1)
      s.tag[i] = TAG_WALL;
    else
      s.tag[i] = owner_of<LBM_MAX_SPHERES>(ss.sph, ss.nsph, x, y, z) >= 0 ? TAG_SOLID : TAG_FLUID;
  }
}
template <class PopT>
__global__ void k_retag_box(Scene<PopT, typename Prec<PopT>::Real> s, const Plan *__restrict__ P) {
  retag_box_body<PopT>(s, P, blockIdx.x, gridDim.x);
}

// Count fresh (FLUID, was SOLID) and dead (SOLID, was FLUID) cells per chunk
// of the box's linear (scan) order.
constexpr int COMPACT_CHUNK = 2048;
constexpr int COMPACT_THREADS = 256;
// Most CTAs a box sweep (retag, compaction) launches: the kernels stride over
// the box or its chunks, so a step whose planned box is small does not pay
// for the empty CTAs of a launch sized for the largest possible box.
constexpr unsigned SWEEP_CTAS = 148 * 4;

__device__ __forceinline__ void box_cell(const Box &bx, long long l, int &x, int &y, int &z) {
  int dx = bx.hi[0] - bx.lo[0] + 1, dy = bx.hi[1] - bx.lo[1] + 1;
  x = bx.lo[0] + (int)(l % dx);
  y = bx.lo[1] + (int)((l / dx) % dy);
  z = bx.lo[2] + (int)(l / ((long long)dx * dy));
}

__device__ __forceinline__ void compact_count_body(const uint8_t *tag, const uint8_t *tagPrev, int nx, int ny,
                                                   const Plan *__restrict__ P, int2 *counts, unsigned bid,
                                                   unsigned gdim) {
  __shared__ int sf[COMPACT_THREADS / 32], sd[COMPACT_THREADS / 32];
  const Box bx = P->U;
  const long long total = P->ucells;
  const int nchunks = P->nchunks;
  // CTAs stride over the chunks (block-uniform trip count)
  for (int c = bid; c < nchunks; c += gdim) {
    const long long base = (long long)c * COMPACT_CHUNK;
    int nf = 0, nd = 0;
    for (int j = threadIdx.x; j < COMPACT_CHUNK; j += blockDim.x) {
      long long l = base + j;
      if (l >= total) break;
      int x, y, z;
      box_cell(bx, l, x, y, z);
      long long i = cell_index(x, y, z, nx, ny);
      uint8_t t = tag[i], p = tagPrev[i];
      nf += (t == TAG_FLUID && p == TAG_SOLID);
      nd += (t == TAG_SOLID && p == TAG_FLUID);
    }
    for (int o = 16; o > 0; o >>= 1) {
      nf += __shfl_xor_sync(0xffffffffu, nf, o);
      nd += __shfl_xor_sync(0xffffffffu, nd, o);
    }
    if ((threadIdx.x & 31) == 0) {
      sf[threadIdx.x >> 5] = nf;
      sd[threadIdx.x >> 5] = nd;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int a = 0, b = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
        a += sf[w];
        b += sd[w];
      }
      counts[c] = make_int2(a, b);
    }
    __syncthreads();  // sf / sd are rewritten for the next chunk
  }
}
static __global__ void k_compact_count(const uint8_t *tag, const uint8_t *tagPrev, int nx, int ny,
                                       const Plan *__restrict__ P, int2 *counts) {
  compact_count_body(tag, tagPrev, nx, ny, P, counts, blockIdx.x, gridDim.x);
}

// Exclusive scan of the per-chunk counts (single CTA, sequential per thread).
__device__ __forceinline__ void compact_scan_body(int2 *counts, const Plan *__restrict__ P, int *totals) {
  __shared__ int2 part[1024];
  const int nchunks = P->nchunks;
  int per = (nchunks + blockDim.x - 1) / blockDim.x;
  int b0 = threadIdx.x * per, b1 = min(b0 + per, nchunks);
  int2 sum = make_int2(0, 0);
  for (int b = b0; b < b1; b++) {
    sum.x += counts[b].x;
    sum.y += counts[b].y;
  }
  part[threadIdx.x] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    int2 run = make_int2(0, 0);
    for (int t = 0; t < (int)blockDim.x; t++) {
      int2 v = part[t];
      part[t] = run;
      run.x += v.x;
      run.y += v.y;
    }
    totals[0] = run.x;
    totals[1] = run.y;
  }
  __syncthreads();
  int2 run = part[threadIdx.x];
  for (int b = b0; b < b1; b++) {
    int2 v = counts[b];
    counts[b] = run;
    run.x += v.x;
    run.y += v.y;
  }
}
static __global__ void k_compact_scan(int2 *counts, const Plan *__restrict__ P, int *totals) {
  compact_scan_body(counts, P, totals);
}

// Emit the fresh / dead cell indices in scan order.
__device__ __forceinline__ void compact_emit_body(const uint8_t *tag, const uint8_t *tagPrev, int nx, int ny,
                                                  const Plan *__restrict__ P, const int2 *offsets, int *fresh,
                                                  int *dead, int cap, unsigned bid, unsigned gdim) {
  __shared__ int wf[COMPACT_THREADS / 32], wd[COMPACT_THREADS / 32];
  __shared__ int runF, runD;
  const Box bx = P->U;
  const long long total = P->ucells;
  const int nchunks = P->nchunks;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  // CTAs stride over the chunks (block-uniform trip count); the inner loop
  // ends on a barrier, so runF / runD are free to be reset for the next chunk
  for (int c = bid; c < nchunks; c += gdim) {
    const long long base = (long long)c * COMPACT_CHUNK;
    if (threadIdx.x == 0) {
      runF = offsets[c].x;
      runD = offsets[c].y;
    }
    __syncthreads();
    for (int j0 = 0; j0 < COMPACT_CHUNK; j0 += blockDim.x) {
      long long l = base + j0 + threadIdx.x;
      bool isF = false, isD = false;
      long long i = 0;
      if (l < total && j0 + (int)threadIdx.x < COMPACT_CHUNK) {
        int x, y, z;
        box_cell(bx, l, x, y, z);
        i = cell_index(x, y, z, nx, ny);
        uint8_t t = tag[i], p = tagPrev[i];
        isF = (t == TAG_FLUID && p == TAG_SOLID);
        isD = (t == TAG_SOLID && p == TAG_FLUID);
      }
      unsigned bf = __ballot_sync(0xffffffffu, isF), bd = __ballot_sync(0xffffffffu, isD);
      if (lane == 0) {
        wf[warp] = __popc(bf);
        wd[warp] = __popc(bd);
      }
      __syncthreads();
      int offF = runF, offD = runD;
      for (int w = 0; w < warp; w++) {
        offF += wf[w];
        offD += wd[w];
      }
      unsigned below = (1u << lane) - 1u;
      if (isF) {
        int pos = offF + __popc(bf & below);
        if (pos < cap) fresh[pos] = (int)i;
      }
      if (isD) {
        int pos = offD + __popc(bd & below);
        if (pos < cap) dead[pos] = (int)i;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        int a = 0, b = 0;
        for (int w = 0; w < nw; w++) {
          a += wf[w];
          b += wd[w];
        }
        runF += a;
        runD += b;
      }
      __syncthreads();
    }
  }
}
static __global__ void k_compact_emit(const uint8_t *tag, const uint8_t *tagPrev, int nx, int ny,
                                      const Plan *__restrict__ P, const int2 *offsets, int *fresh,
                                      int *dead, int cap) {
  compact_emit_body(tag, tagPrev, nx, ny, P, offsets, fresh, dead, cap, blockIdx.x, gridDim.x);
}

// One fresh cell (src/sim.js:264-308): the FLUID neighbours' phi, rho and u
// averaged in the reference's neighbour order (dz, dy, dx ascending), then phi,
// phiPrev, rho, u and the equilibrium populations written.  nb(j, p, r, x, y,
// z) gives neighbour j's five values.
template <class PopT, class NB>
__device__ __forceinline__ void fill_cell(const Scene<PopT, typename Prec<PopT>::Real> &s, int cur, long long i,
                                          double rhoL, double rhoG, NB &&nb) {
  using Real = typename Prec<PopT>::Real;
  const int nx = s.nx, ny = s.ny;
  double psum = 0, rsum = 0, vxs = 0, vys = 0, vzs = 0;
  int pcnt = 0;
  for (int dz = -1; dz <= 1; dz++)
    for (int dy = -1; dy <= 1; dy++)
      for (int dx = -1; dx <= 1; dx++) {
        if (!dx && !dy && !dz) continue;
        long long j = i + ((long long)dz * ny + dy) * nx + dx;
        if (s.tag[j] == TAG_FLUID) {
          Real vp, vr, vx_, vy_, vz_;
          nb(j, vp, vr, vx_, vy_, vz_);
          psum += (double)vp;
          rsum += (double)vr;
          vxs += (double)vx_;
          vys += (double)vy_;
          vzs += (double)vz_;
          pcnt++;
        }
      }
  double p = pcnt > 0 ? psum / pcnt : (double)s.phi[cur][i];
  double r = pcnt > 0 ? rsum / pcnt : 1.0;
  double vx = pcnt > 0 ? vxs / pcnt : 0;
  double vy = pcnt > 0 ? vys / pcnt : 0;
  double vz = pcnt > 0 ? vzs / pcnt : 0;
  Real pR = (Real)p;
  s.phi[cur][i] = pR;
  s.phi[1 - cur][i] = pR;  // phiPrev[i] = p
  s.rho[cur][i] = (Real)r;
  s.set_ux(cur, i, (Real)vx);
  s.set_uy(cur, i, (Real)vy);
  s.uz[cur][i] = (Real)vz;
  double rhoPhase = rhoG + p * (rhoL - rhoG);
  double u2 = vx * vx + vy * vy + vz * vz;
  for (int k = 0; k < Q27; k++) {
    double eu = dcomp(k, 0) * vx + dcomp(k, 1) * vy + dcomp(k, 2) * vz;
    double Qi = eu * (3.0 + 4.5 * eu) - 1.5 * u2;
    double fk = (double)w27_of(k) * (r + rhoPhase * Qi);
    s.F[cur][pidx<27>(k, i)] = Codec<PopT>::enc((Real)fk, (Real)w27_of(k));
  }
  for (int k = 0; k < Q7; k++) {
    double eu = dcomp(k, 0) * vx + dcomp(k, 1) * vy + dcomp(k, 2) * vz;
    double hk = (double)w7_of(k) * p * (1 + 4.0 * eu);
    s.H[cur][pidx<7>(k, i)] = Codec<PopT>::enc((Real)hk, (Real)w7_of(k) * pR);
  }
}

// Fresh cells a block fills in parallel; a longer list is filled by one
// thread in list order.
constexpr int FILL_PAR_MAX = 512;
constexpr int FILL_THREADS = 256;

// handleFreshCells over the scan-ordered fresh list (src/sim.js:257-310).  The
// reference fills in scan order, in place: a fresh cell sees the filled values
// of fresh neighbours before it in scan order and the old values of those
// after it.  In parallel that order is kept by rounds: the old phi, rho and u
// of every listed cell are saved first; in each round a cell whose fresh
// neighbours before it in scan order were all filled in earlier rounds is
// filled, reading the saved old values for fresh neighbours after it.  The
// arithmetic of each cell is the sequential one (fill_cell), so the results
// are the same bit for bit.  A z slab fills its own planes only (its copied
// planes receive the neighbouring slab's filled values).  sequential != 0: one
// thread in list order (also used for lists longer than FILL_PAR_MAX).
template <class PopT>
__device__ __forceinline__ void fresh_fill_body(const Scene<PopT, typename Prec<PopT>::Real> &s, int cur,
                                                const int *fresh, const int *totals, int cap, double rhoL,
                                                double rhoG, int zlo, int zend, int sequential) {
  using Real = typename Prec<PopT>::Real;
  int nf = totals[0];
  if (nf > cap) nf = cap;
  const long long nxny = (long long)s.nx * s.ny;
  auto skip = [&](long long i) -> bool {
    if (zend <= 0) return false;
    const long long z = i / nxny;
    return z < zlo || z >= zend;
  };
  auto current = [&](long long j, Real &p, Real &r, Real &x, Real &y, Real &z) {
    p = s.phi[cur][j];
    r = s.rho[cur][j];
    x = s.ux_at(cur, j);
    y = s.uy_at(cur, j);
    z = s.uz[cur][j];
  };
  if (sequential || nf > FILL_PAR_MAX) {
    if (threadIdx.x != 0) return;
    for (int q = 0; q < nf; q++) {
      const long long i = fresh[q];
      if (!skip(i)) fill_cell<PopT>(s, cur, i, rhoL, rhoG, current);
    }
    return;
  }
  __shared__ int sIdx[FILL_PAR_MAX];
  __shared__ int sDone[FILL_PAR_MAX];  // round in which the cell was filled (or skipped), 0: not yet
  __shared__ Real sOld[5][FILL_PAR_MAX];
  for (int q = threadIdx.x; q < nf; q += blockDim.x) {
    const long long i = fresh[q];
    sIdx[q] = (int)i;
    sDone[q] = 0;
    current(i, sOld[0][q], sOld[1][q], sOld[2][q], sOld[3][q], sOld[4][q]);
  }
  __syncthreads();
  // list position of cell j, or -1 (the list is sorted by cell index)
  auto find = [&](long long j) -> int {
    int lo = 0, hi = nf - 1;
    while (lo <= hi) {
      const int mid = (lo + hi) >> 1;
      const int v = sIdx[mid];
      if (v == j) return mid;
      if (v < j) lo = mid + 1;
      else hi = mid - 1;
    }
    return -1;
  };
  for (int round = 1;; round++) {
    int waiting = 0;
    for (int q = threadIdx.x; q < nf; q += blockDim.x) {
      if (sDone[q]) continue;
      const long long i = sIdx[q];
      if (skip(i)) {
        sDone[q] = round;
        continue;
      }
      bool ready = true;
      for (int dz = -1; dz <= 0 && ready; dz++)
        for (int dy = -1; dy <= 1 && ready; dy++)
          for (int dx = -1; dx <= 1; dx++) {
            if (dz == 0 && (dy > 0 || (dy == 0 && dx >= 0))) break;  // only neighbours before i
            const long long j = i + ((long long)dz * s.ny + dy) * s.nx + dx;
            const int pos = find(j);
            if (pos >= 0 && (sDone[pos] == 0 || sDone[pos] >= round)) {
              ready = false;
              break;
            }
          }
      if (!ready) {
        waiting = 1;
        continue;
      }
      fill_cell<PopT>(s, cur, i, rhoL, rhoG, [&](long long j, Real &p, Real &r, Real &x, Real &y, Real &z) {
        const int pos = j > i ? find(j) : -1;
        if (pos >= 0) {
          p = sOld[0][pos];
          r = sOld[1][pos];
          x = sOld[2][pos];
          y = sOld[3][pos];
          z = sOld[4][pos];
        } else {
          current(j, p, r, x, y, z);
        }
      });
      sDone[q] = round;
    }
    if (!__syncthreads_or(waiting)) break;
  }
}
template <class PopT>
__global__ void __launch_bounds__(FILL_THREADS)
    k_fresh_fill(Scene<PopT, typename Prec<PopT>::Real> s, int cur, const int *fresh, const int *totals, int cap,
                 double rhoL, double rhoG, int zlo, int zend, int sequential) {
  if (blockIdx.x != 0) return;
  fresh_fill_body<PopT>(s, cur, fresh, totals, cap, rhoL, rhoG, zlo, zend, sequential);
}

// absorbDeadCells (src/solid.js:87-101): impulse rho(phi)*u of every cell on
// the scan-ordered dead list, in FP64, to the sphere owning the cell.  One CTA
// per sphere; thread t sums the contiguous t-th share of the list in scan
// order, then a fixed shared-memory tree adds the shares -- deterministic,
// and independent of how many dead cells there are per step.
// ---------------------------------------------------------------- generic solids
// retagCells(solid) for any duck-typed solid (src/sim.js:214-244): the host
// has evaluated solid.contains / solid.surfaceVelocity per cell into mask
// (non-zero = inside) and us (3 floats per cell, x y z; null = at rest).
template <class PopT>
__global__ void k_retag_mask(Scene<PopT, typename Prec<PopT>::Real> s, int cur, const uint8_t *__restrict__ mask,
                             const float *__restrict__ us) {
  using Real = typename Prec<PopT>::Real;
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= s.n) return;
  const int nx = s.nx, ny = s.ny, nz = s.nz;
  int x = (int)(i % nx);
  long long t = i / nx;
  int y = (int)(t % ny);
  int z = (int)(t / ny);
  s.tagPrev[i] = s.tag[i];
  s.phi[1 - cur][i] = s.phi[cur][i];
  if (x == 0 || x == nx - 1 || y == 0 || y == ny - 1 || z == 0 || z == nz - 1) {
    s.tag[i] = TAG_WALL;
    s.usx[i] = s.usy[i] = s.usz[i] = (Real)0;
  } else if (mask[i]) {
    s.tag[i] = TAG_SOLID;
    s.usx[i] = us ? (Real)us[3 * i] : (Real)0;
    s.usy[i] = us ? (Real)us[3 * i + 1] : (Real)0;
    s.usz[i] = us ? (Real)us[3 * i + 2] : (Real)0;
  } else {
    s.tag[i] = TAG_FLUID;
    s.usx[i] = s.usy[i] = s.usz[i] = (Real)0;
  }
}

// Momentum-exchange links of the last hydro stream (after
// k_stream_hydro_macro, while F[1 - cur] still holds the post-collision f2):
// for every interior FLUID cell i in scan order and every direction k whose
// source i - e_k is SOLID, the link (i, k, m) with m = f2_opp(i) + f_k(i), the
// value src/sim.js:529-531 hands to solid.applyImpulseAtCell (as
// -m e_k at the solid cell).  Three passes: count per chunk, scan, emit.
constexpr int LINK_CHUNK = 1024;  // cells per chunk = threads per block

__device__ __forceinline__ uint32_t solid_links(const uint8_t *tag, long long i, int nx, int ny, int nz) {
  if (tag[i] != TAG_FLUID || !interior_cell(i, nx, ny, nz)) return 0u;
  uint32_t m = 0;
  for (int k = 1; k < Q27; k++) {
    const long long src = i - (((long long)dcomp(k, 2) * ny + dcomp(k, 1)) * nx + dcomp(k, 0));
    if (tag[src] == TAG_SOLID) m |= 1u << k;
  }
  return m;
}

__device__ __forceinline__ int block_exclusive_scan(int v, int *sh, int &total) {
  // Hillis-Steele over one block of LINK_CHUNK threads
  const int t = threadIdx.x;
  sh[t] = v;
  __syncthreads();
  for (int d = 1; d < LINK_CHUNK; d <<= 1) {
    const int a = t >= d ? sh[t - d] : 0;
    __syncthreads();
    sh[t] += a;
    __syncthreads();
  }
  total = sh[LINK_CHUNK - 1];
  const int excl = sh[t] - v;
  __syncthreads();
  return excl;
}

static __global__ void __launch_bounds__(LINK_CHUNK) k_link_count(const uint8_t *tag, int nx, int ny, int nz,
                                                                 long long n, int *chunkCount) {
  __shared__ int sh[LINK_CHUNK];
  const long long i = (long long)blockIdx.x * LINK_CHUNK + threadIdx.x;
  const int c = i < n ? __popc(solid_links(tag, i, nx, ny, nz)) : 0;
  int total;
  block_exclusive_scan(c, sh, total);
  if (threadIdx.x == 0) chunkCount[blockIdx.x] = total;
}

// exclusive scan of the chunk counts in place; total into chunkCount[nchunks]
static __global__ void k_link_scan(int *chunkCount, int nchunks) {
  __shared__ int part[1024];
  const int per = (nchunks + blockDim.x - 1) / blockDim.x;
  const int b0 = threadIdx.x * per, b1 = min(b0 + per, nchunks);
  int sum = 0;
  for (int b = b0; b < b1; b++) sum += chunkCount[b];
  part[threadIdx.x] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int t = 0; t < (int)blockDim.x; t++) {
      const int v = part[t];
      part[t] = run;
      run += v;
    }
    chunkCount[nchunks] = run;
  }
  __syncthreads();
  int run = part[threadIdx.x];
  for (int b = b0; b < b1; b++) {
    const int v = chunkCount[b];
    chunkCount[b] = run;
    run += v;
  }
}

template <class PopT>
__global__ void __launch_bounds__(LINK_CHUNK) k_link_emit(Scene<PopT, typename Prec<PopT>::Real> s, int cur,
                                                         const int *chunkOff, int cap, int *cells,
                                                         int8_t *dirs, double *mom) {
  __shared__ int sh[LINK_CHUNK];
  const long long i = (long long)blockIdx.x * LINK_CHUNK + threadIdx.x;
  const uint32_t m = i < s.n ? solid_links(s.tag, i, s.nx, s.ny, s.nz) : 0u;
  int total;
  int pos = chunkOff[blockIdx.x] + block_exclusive_scan(__popc(m), sh, total);
  const PopT *f2 = s.F[1 - cur];
  const PopT *f = s.F[cur];
  for (uint32_t r = m; r; r &= r - 1, pos++) {
    const int k = __ffs(r) - 1;
    if (pos >= cap) break;
    const double fopp = (double)Codec<PopT>::dec(f2[pidx<27>(opp_of(k), i)], 0);
    const double fk = (double)Codec<PopT>::dec(f[pidx<27>(k, i)], 0);
    cells[pos] = (int)i;
    dirs[pos] = (int8_t)k;
    mom[pos] = fopp + fk;
  }
}

constexpr int DEAD_THREADS = 256;

// (static: Real = float is instantiated by several translation units)
// the dead-cell sweep reads phi and u through one of these: plain arrays
// (the allocation-free entry's caller arrays) or a scene's current half
template <class Real>
struct ArrayFields {
  const Real *phi, *ux, *uy, *uz;
  __device__ __forceinline__ double p(long long i) const { return (double)phi[i]; }
  __device__ __forceinline__ double vx(long long i) const { return (double)ux[i]; }
  __device__ __forceinline__ double vy(long long i) const { return (double)uy[i]; }
  __device__ __forceinline__ double vz(long long i) const { return (double)uz[i]; }
};
template <class PopT>
struct SceneFields {
  const Scene<PopT, typename Prec<PopT>::Real> &s;
  int cur;
  __device__ __forceinline__ double p(long long i) const { return (double)s.phi[cur][i]; }
  __device__ __forceinline__ double vx(long long i) const { return (double)s.ux_at(cur, i); }
  __device__ __forceinline__ double vy(long long i) const { return (double)s.uy_at(cur, i); }
  __device__ __forceinline__ double vz(long long i) const { return (double)s.uz[cur][i]; }
};

template <class Fields>
__device__ __forceinline__ void absorb_dead_body(const Fields &fd, int nx, int ny, const int *__restrict__ dead,
                                                 const int *__restrict__ totals, int cap, double rhoL,
                                                 double rhoG, const SolidSet *__restrict__ ssp, double *out,
                                                 int b) {
  __shared__ double sh[6][DEAD_THREADS];
  const SolidSet &ss = *ssp;
  if (b >= ss.nsph) return;
  int nd = totals[1];
  if (nd > cap) nd = cap;
  const double dRho = rhoL - rhoG;
  const int per = (nd + DEAD_THREADS - 1) / DEAD_THREADS;
  const int q0 = threadIdx.x * per, q1 = min(q0 + per, nd);
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int q = q0; q < q1; q++) {
    const long long i = dead[q];
    const int x = (int)(i % nx);
    const long long t = i / nx;
    const int y = (int)(t % ny);
    const int z = (int)(t / ny);
    if (ss.zend > 0 && (z < ss.zlo || z >= ss.zend)) continue;
    if (owner_of<LBM_MAX_SPHERES>(ss.sph, ss.nsph, x, y, z) != b) continue;
    const double rhoPhase = __dadd_rn(rhoG, __dmul_rn(fd.p(i), dRho));
    impulse_terms(ss.sph[b], x, y, z, __dmul_rn(rhoPhase, fd.vx(i)), __dmul_rn(rhoPhase, fd.vy(i)),
                  __dmul_rn(rhoPhase, fd.vz(i)), acc);
  }
  for (int j = 0; j < 6; j++) sh[j][threadIdx.x] = acc[j];
  __syncthreads();
  for (int st = DEAD_THREADS / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st)
      for (int j = 0; j < 6; j++) sh[j][threadIdx.x] = __dadd_rn(sh[j][threadIdx.x], sh[j][threadIdx.x + st]);
    __syncthreads();
  }
  if (threadIdx.x < 6) out[6 * b + threadIdx.x] = sh[threadIdx.x][0];
}
template <class Real>
static __global__ void __launch_bounds__(DEAD_THREADS)
    k_absorb_dead(const Real *__restrict__ phi, const Real *__restrict__ ux,
                  const Real *__restrict__ uy, const Real *__restrict__ uz, int nx, int ny,
                  const int *__restrict__ dead, const int *__restrict__ totals, int cap, double rhoL,
                  double rhoG, const SolidSet *__restrict__ ssp, double *out) {
  absorb_dead_body(ArrayFields<Real>{phi, ux, uy, uz}, nx, ny, dead, totals, cap, rhoL, rhoG, ssp, out,
                   blockIdx.x);
}
// the same over a scene's current half
template <class PopT>
static __global__ void __launch_bounds__(DEAD_THREADS)
    k_absorb_dead_scene(Scene<PopT, typename Prec<PopT>::Real> s, int cur, const int *__restrict__ dead,
                        const int *__restrict__ totals, int cap, double rhoL, double rhoG,
                        const SolidSet *__restrict__ ssp, double *out) {
  absorb_dead_body(SceneFields<PopT>{s, cur}, s.nx, s.ny, dead, totals, cap, rhoL, rhoG, ssp, out, blockIdx.x);
}

// Deterministic reduction of the per-cell impulse arrays in one launch.
// Block (c, b) sums chunk c (1024 cells) of sphere b's slots -- the threads
// stride the chunk, then a shared-memory tree -- zeroes the slots it read (so
// the next step starts from zero without a clearing launch) and stores its
// partial; the block that takes the last ticket of sphere b adds the partials
// in chunk order and resets the ticket.  Which block finishes last does not
// change the result, nor does how the stream kernel was tiled.
constexpr int RED_CHUNK = 1024;
constexpr int RED_THREADS = 256;

__device__ __forceinline__ void impulse_reduce_body(const SolidSet *__restrict__ ssp, double *partials,
                                                    int maxChunks, double *out, unsigned *tickets, int cx,
                                                    int b) {
  const SolidSet &ss = *ssp;
  if (b >= ss.nsph) return;
  const ImpulseTarget &t = ss.imp[b];
  const long long cells = (long long)t.dim[0] * t.dim[1] * t.dim[2];
  int nch = (int)((cells + RED_CHUNK - 1) / RED_CHUNK);
  if (nch < 1) nch = 1;  // an empty box still gives its zero
  if (nch > maxChunks) nch = maxChunks;
  if (cx >= nch) return;
  const long long c0 = (long long)cx * RED_CHUNK;
  __shared__ double sh[6][RED_THREADS];
  __shared__ bool last;
  // Only cells within sqrt(3) outside the sphere hold links (a FLUID cell next
  // to one the sphere contains); the rest of the box stays zero and is
  // neither read nor cleared.  Skipping a +0 term does not change a sum.
  const SphereDesc &sp = ss.sph[b];
  const double rIn = sp.r > 1.0 ? sp.r - 1.0 : 0.0, rOut = sp.r + 2.0;
  const double in2 = rIn * rIn, out2 = rOut * rOut;
  const int dxb = t.dim[0], dyb = t.dim[1];
  double a[6] = {0, 0, 0, 0, 0, 0};
  for (int j = threadIdx.x; j < RED_CHUNK; j += RED_THREADS) {
    const long long c = c0 + j;
    if (c >= cells) break;
    const int lx = (int)(c % dxb), ly = (int)((c / dxb) % dyb), lz = (int)(c / ((long long)dxb * dyb));
    const double ex = t.lo[0] + lx + 0.5 - sp.cx, ey = t.lo[1] + ly + 0.5 - sp.cy, ez = t.lo[2] + lz + 0.5 - sp.cz;
    const double d2 = ex * ex + ey * ey + ez * ez;
    if (d2 < in2 || d2 > out2) continue;
    double *p = t.acc + 6 * c;
    for (int q = 0; q < 6; q++) a[q] = __dadd_rn(a[q], p[q]);
    for (int q = 0; q < 6; q++) p[q] = 0.0;
  }
  for (int q = 0; q < 6; q++) sh[q][threadIdx.x] = a[q];
  __syncthreads();
  for (int st = RED_THREADS / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st)
      for (int q = 0; q < 6; q++) sh[q][threadIdx.x] = __dadd_rn(sh[q][threadIdx.x], sh[q][threadIdx.x + st]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    for (int q = 0; q < 6; q++) partials[((long long)b * maxChunks + cx) * 6 + q] = sh[q][0];
    __threadfence();
    last = atomicAdd(&tickets[b], 1u) == (unsigned)nch - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (threadIdx.x < 6) {
    double s = 0;
    for (int c = 0; c < nch; c++) s = __dadd_rn(s, __ldcg(&partials[((long long)b * maxChunks + c) * 6 + threadIdx.x]));
    out[6 * b + threadIdx.x] = s;
  }
  if (threadIdx.x == 0) tickets[b] = 0;
}
static __global__ void __launch_bounds__(RED_THREADS)
    k_impulse_reduce(const SolidSet *__restrict__ ssp, double *partials, int maxChunks, double *out,
                     unsigned *tickets) {
  impulse_reduce_body(ssp, partials, maxChunks, out, tickets, blockIdx.x, blockIdx.y);
}

// Device-side plan for the device-resident loop: sphere descriptors from the
// device sphere state, the retag box (current and two previous sphere boxes),
// compaction chunking, and impulse slots of slotCells cells per sphere.
__device__ __forceinline__ void plan_body(Plan *P, const lbm_sphere *sph, int nsph, int nx, int ny, int nz,
                                          double *impBase, long long slotCells, long long maxUCells) {
  if (threadIdx.x != 0) return;
  SolidSet &ss = P->ss;
  ss.nsph = nsph;
  Box now{{1, 1, 1}, {0, 0, 0}};
  int redChunks = 1;
  for (int b = 0; b < nsph; b++) {
    SphereDesc &d = ss.sph[b];
    d.cx = sph[b].cx;
    d.cy = sph[b].cy;
    d.cz = sph[b].cz;
    d.r = sph[b].r;
    d.vx = sph[b].vx;
    d.vy = sph[b].vy;
    d.vz = sph[b].vz;
    d.wx = sph[b].wx;
    d.wy = sph[b].wy;
    d.wz = sph[b].wz;
    Box sb = sphere_box(d.cx, d.cy, d.cz, d.r, nx, ny, nz);
    now = box_union(now, sb);
    Box tb = box_grow(sb, 1, nx, ny, nz);
    ImpulseTarget &t = ss.imp[b];
    t.acc = impBase + (long long)b * slotCells * 6;
    long long cells = box_cells(tb);
    if (cells > slotCells) {
      P->overflow = 1;
      cells = 0;
      tb = Box{{1, 1, 1}, {0, 0, 0}};
    }
    for (int a = 0; a < 3; a++) {
      t.lo[a] = box_empty(tb) ? 0 : tb.lo[a];
      t.dim[a] = box_empty(tb) ? 0 : tb.hi[a] - tb.lo[a] + 1;
    }
    int rc = (int)((cells + RED_CHUNK - 1) / RED_CHUNK);
    redChunks = rc > redChunks ? rc : redChunks;
  }
  Box U;
  if (P->fullRetag > 0) {
    U = Box{{0, 0, 0}, {nx - 1, ny - 1, nz - 1}};
    P->fullRetag--;
  } else {
    U = box_union(box_union(now, P->boxLast), P->boxLastLast);
  }
  long long uc = box_cells(U);
  if (uc > maxUCells) {
    P->overflow = 1;
    uc = 0;
    U = Box{{1, 1, 1}, {0, 0, 0}};
  }
  P->U = U;
  P->ucells = uc;
  P->nchunks = (int)((uc + COMPACT_CHUNK - 1) / COMPACT_CHUNK);
  P->redChunks = redChunks;
  P->impDoubles = (long long)nsph * slotCells * 6;
  P->boxLastLast = P->boxLast;
  P->boxLast = now;
}
static __global__ void k_plan(Plan *P, const lbm_sphere *sph, int nsph, int nx, int ny, int nz,
                              double *impBase, long long slotCells, long long maxUCells) {
  if (blockIdx.x != 0) return;
  plan_body(P, sph, nsph, nx, ny, nz, impBase, slotCells, maxUCells);
}

// packVolume's two bytes of cell i (src/sim.js:586-600): R = clamp01(phi) *
// 255 truncated (a NaN gives 0), G = 255 for a SOLID cell, else 0
template <class Real>
__device__ __forceinline__ void pack_rg8(uint8_t *out, long long i, Real phi, bool solid) {
  double p = (double)phi;
  if (p < 0.0) p = 0.0;
  else if (p > 1.0) p = 1.0;
  const double v = p * 255.0;
  uchar2 o;
  o.x = (uint8_t)((v == v) ? (int)v : 0);
  o.y = solid ? 255 : 0;
  reinterpret_cast<uchar2 *>(out)[i] = o;
}

// packVolume (src/sim.js:586-600)
template <class PopT>
__global__ void k_pack(Scene<PopT, typename Prec<PopT>::Real> s, int cur, uint8_t *out) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= s.n) return;
  pack_rg8(out, i, s.phi[cur][i], s.tag[i] == TAG_SOLID);
}

// packVolume of the planes z = 0 and z = nz - 1 only: the fused step packs
// every other cell on a frame step
template <class PopT>
__global__ void k_pack_end_planes(Scene<PopT, typename Prec<PopT>::Real> s, int cur, uint8_t *out) {
  const long long plane = (long long)s.nx * s.ny;
  long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (j >= 2 * plane) return;
  const long long i = j < plane ? j : (long long)(s.nz - 1) * plane + (j - plane);
  pack_rg8(out, i, s.phi[cur][i], s.tag[i] == TAG_SOLID);
}

// NaN/Inf watchdog: the lowest index of a cell whose phi, rho or u is not
// finite is min-ed into *first, which the caller sets to ~0 beforehand (rho
// alone would not do: rho = sum f > 0.01 ? sum f : 0.01 turns a NaN sum into
// 0.01, src/sim.js:546).  The loop strides by whole blocks, so every warp
// takes the same trips and one lane per warp that sees such a cell does the
// atomic.
template <class PopT>
__global__ void k_watch_finite(Scene<PopT, typename Prec<PopT>::Real> s, int cur, unsigned long long *first) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i0 = blockIdx.x * (long long)blockDim.x; i0 < s.n; i0 += stride) {
    const long long i = i0 + threadIdx.x;
    bool bad = false;
    if (i < s.n)
      bad = !isfinite((double)s.phi[cur][i]) || !isfinite((double)s.rho[cur][i]) ||
            !isfinite((double)s.ux_at(cur, i)) || !isfinite((double)s.uy_at(cur, i)) ||
            !isfinite((double)s.uz[cur][i]);
    const unsigned m = __ballot_sync(0xffffffffu, bad);
    if (m && (int)(threadIdx.x & 31) == __ffs(m) - 1) atomicMin(first, (unsigned long long)i);
  }
}

}  // namespace lbm
