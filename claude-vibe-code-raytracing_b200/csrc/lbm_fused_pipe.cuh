// The compact-ring forms of the fused LBM step (tile shapes 4 or 6 rows |
// LBM_FUSED_COMPACT, LBM_FUSED_ASYNC or LBM_FUSED_STAGED; 6 rows |
// LBM_FUSED_TMA).
//
// Same algorithm and arithmetic as fused_tile (lbm_fused.cuh): a CTA owns a
// 32 x TY column of cells and marches it up a z-chunk; each plane is collided
// at its source into a shared-memory ring and pulled from there.  What
// differs is the ring and how the data reach the SM:
//
//   * the ring stores, for each direction, only the cells that can be a
//     source of that direction for the tile plus the tile itself for
//     bounce-back (33 columns by TY or TY + 1 rows), so a cell's index in any
//     direction's array is one per-thread term plus a compile-time constant:
//     46 KB at 4 rows (three CTAs per SM), 66 KB at 6 rows (two);
//   * the halo rows and columns are collided by two halo warps (the rows above
//     and below; the side columns with the corners, one half-warp per side),
//     which load right after the barrier that ends a plane, while the cell
//     warps pull it, so their latency is off the critical path;
//   * the cell warps' loads of the next plane:
//       - COMPACT: plain loads into registers at the start of each plane;
//       - ASYNC: each thread copies its own cell of plane q + 1 (populations
//         by whole groups, rho, u and the phi stencil) into its own
//         shared-memory slots with per-thread asynchronous copies issued
//         after it has written plane q into the ring, so the copies land
//         while plane q - 1 is pulled and no registers are held meanwhile;
//       - STAGED: the tile rows of plane q + 1 arrive by bulk asynchronous
//         copies (cp.async.bulk, completion counted in bytes on an mbarrier)
//         issued by one producer lane as soon as every cell warp has read the
//         current stage (a second mbarrier);
//       - TMA: the same stage (rows of plane q + 1, phi of plane q + 2) as
//         six to eight tensor-map box copies (the tile's 4 population blocks
//         x 6 rows of f and of h, the rho / u / tag rows, the phi rows with
//         their halo), issued by one lane of the halo-row warp right after
//         the barrier that follows the cell warps' reads of the stage, so the
//         copies land while plane q is emitted and plane q - 1 pulled and no
//         cell warp waits on a load it issued.
//         Needs nx a multiple of 16 (whole blocks per tile row, 16-byte row
//         strides of the tags).
//       - L2PF: the COMPACT loads; in addition, one lane of the halo-row warp
//         asks the tensor-copy unit, right after the first barrier of plane
//         q, to bring the tile's rows of plane q + 2 (FP16/BF16: q + 3):
//         f, h, rho, u, tags, and phi with its halo rows one plane further,
//         into L2.  Nothing is staged in shared memory and nothing is waited
//         on: the cell and halo warps' own loads then find their lines in
//         L2.  Same tensor maps and coordinates as TMA.
//
// Results are bit-identical to fused_tile in every form (the collision is the
// same collide_cell, the pull sums in the same order).  FP32, FP16 and BF16
// storage; the waits for the bulk stage are bounded like every other wait of
// the library (status word + fault code 90 + LBM_ERR_TIMEOUT).
#pragma once

#include "lbm_fused.cuh"

namespace lbm {

// launch forms of the compact-ring kernel (the FORM of the launch tables)
constexpr int PIPE_STAGED = 1;
constexpr int PIPE_COMPACT = 2;
constexpr int PIPE_ASYNC = 3;
constexpr int PIPE_TMA = 4;
constexpr int PIPE_L2PF = 5;
// planes ahead of the one being collided that the L2-prefetch form asks for
// (measured at 256^3: FP32 2 of 1-4, FP16 3)
template <class PopT>
constexpr int l2pf_ahead() {
  return sizeof(PopT) == 4 ? 2 : 3;
}

// ---------------------------------------------------------------- compact ring
// Direction k's slot array in one ring copy covers the local columns
// [cx0, cx0 + 33) and rows [ry0, ry0 + H) of the tile (local (0, 0) is the
// tile's first cell; -1 and 32 / TY are the halo): a direction with e_x = +1
// is pulled by column 0 from column -1, so its array starts at column -1, and
// so on.  Every tile cell is inside every array (bounce-back reads the cell's
// own value of the opposite direction).  All arrays are 33 wide (one column
// unused where e_x = 0), so a cell's index in any array is the same
// per-thread term ty * 33 + tx plus a compile-time constant.
template <int TY>
struct PipeRing {
  static constexpr int W(int) { return 33; }
  static constexpr int H(int k) { return TY + (kDir[k][1] != 0 ? 1 : 0); }
  static constexpr int CX0(int k) { return kDir[k][0] > 0 ? -1 : 0; }
  static constexpr int RY0(int k) { return kDir[k][1] > 0 ? -1 : 0; }
  static constexpr int S(int k) { return W(k) * H(k); }
  // offset of direction k inside its e_z group (Q = 27 or 7 directions)
  static constexpr int off(int Q, int k) {
    int o = 0;
    for (int j = 0; j < k; j++)
      if (kDir[j][2] == kDir[k][2]) o += S(j);
    return o;
  }
  static constexpr int grp(int Q, int ez) {
    int o = 0;
    for (int j = 0; j < Q; j++)
      if (kDir[j][2] == ez) o += S(j);
    return o;
  }
  // Copies of each e_z group, one per plane whose slots may still be read
  // while the next plane is written.  A plane's e_z = -1 slots are read by
  // the pulls of the plane below and of itself, its e_z = 0 slots by its own
  // pull, its e_z = +1 slots by its own pull and the plane above's, its tags
  // by the pulls of the planes below, at and above it; a barrier separates
  // the pull of plane q - 2 from the writes of plane q, so 2 / 2 / 3 copies
  // and 3 tag planes suffice.
  static constexpr int CM = 2, CZ = 2, CP = 3, CT = 3;
  // f: e_z = -1 group in CM copies, e_z = 0 in CZ, e_z = +1 in CP; h likewise
  static constexpr int FM = 0;
  static constexpr int FZ = FM + CM * grp(27, -1);
  static constexpr int FP = FZ + CZ * grp(27, 0);
  static constexpr int HM = FP + CP * grp(27, 1);
  static constexpr int HZ = HM + CM * grp(7, -1);
  static constexpr int HP = HZ + CZ * grp(7, 0);
  static constexpr int TOTAL = HP + CP * grp(7, 1);
  // index of local cell (lx, ly) in direction k's array, without the copy base
  static constexpr int at(int Q, int k, int lx, int ly) {
    return off(Q, k) + (ly - RY0(k)) * W(k) + (lx - CX0(k));
  }
};
// copy of plane p in a ring of C copies (p >= -C)
template <int C>
__device__ __forceinline__ int ring_copy(int p) {
  return (int)((unsigned)(p + C) % (unsigned)C);
}

// ---------------------------------------------------------------- shared memory
template <class PopT, int TY, int PF>
struct PipeSmem {
  using Real = typename Prec<PopT>::Real;
  static constexpr bool STG = PF == PIPE_STAGED, ASY = PF == PIPE_ASYNC, TMA = PF == PIPE_TMA;
  using R = PipeRing<TY>;
  static constexpr int CT = R::CT;  // tag planes
  static constexpr int RX = 34, RY = TY + 2, NC = RX * RY;  // tag planes keep the full halo frame
  // blocks a 32-cell row can span (4 when rows start on a block: TMA)
  static constexpr int SB = TMA ? 4 : 5;
  static constexpr int ROWF = SB * PopGroups<Q27>::BLOCK, ROWH = SB * PopGroups<Q7>::BLOCK;
  static constexpr int MROW = TMA ? 32 : 36;  // floats of one staged rho / u row (16-byte aligned copy)
  static constexpr int TROW = TMA ? 32 : 48;  // bytes of one staged tag row
  static constexpr int PROW = 40;             // floats of one staged phi row (x0 - 4 .. x0 + 35)
  // floats of one staged phi plane (a 128-byte multiple for the tensor copies)
  static constexpr int PSL = TMA ? ((TY + 2) * PROW + 31) / 32 * 32 : (TY + 2) * PROW;
  // alignment of the stage buffers: tensor-copy destinations are 128-byte
  // aligned (the base itself is aligned up by the tile, see `lead`)
  static constexpr size_t AL = TMA ? 128 : 16;
  static constexpr size_t lead = TMA ? 128 : 0;  // room to align the base up
  static constexpr size_t ringBytes = (size_t)R::TOTAL * sizeof(Real);
  static constexpr size_t tagOff = ringBytes;
  static constexpr size_t stF = (tagOff + CT * NC + AL - 1) / AL * AL;
  static constexpr size_t stH = stF + (size_t)TY * ROWF * sizeof(PopT);
  static constexpr size_t stM = stH + (size_t)TY * ROWH * sizeof(PopT);
  static constexpr size_t stT = stM + (size_t)4 * TY * MROW * sizeof(Real);
  static constexpr size_t phiOff = (stT + (size_t)TY * TROW + AL - 1) / AL * AL;
  static constexpr size_t barOff = (phiOff + (size_t)3 * PSL * sizeof(Real) + 15) / 16 * 16;
  // bytes of one TMA stage: the rows of f, h, rho, uz, the tags (and ux, uy
  // unless they sit in the pad slots), one phi plane; the prologue adds two
  // phi planes
  static constexpr bool UPAD = sizeof(PopT) == sizeof(Real);
  static constexpr uint32_t tmaRows = (uint32_t)(TY * (ROWF + ROWH) * sizeof(PopT) +
                                                 (UPAD ? 2 : 4) * TY * MROW * sizeof(Real) + TY * TROW);
  static constexpr uint32_t tmaPhi = (uint32_t)((TY + 2) * PROW * sizeof(Real));
  // the async form's per-thread slots after the tag planes: [G27][32 TY]
  // groups of f, [G7][32 TY] groups of h, [11][32 TY] words (phi and its six
  // neighbours, rho, ux, uy, uz)
  static constexpr int NT = 32 * TY, GB = 4 * (int)sizeof(PopT), NS = 11;
  static constexpr size_t aF = (tagOff + CT * NC + 15) / 16 * 16;
  static constexpr size_t aH = aF + (size_t)PopGroups<Q27>::G * NT * GB;
  static constexpr size_t aS = aH + (size_t)PopGroups<Q7>::G * NT * GB;
  // staged: two mbarriers (stage full, stage read) and the abort flag (TMA:
  // the first mbarrier only); compact: ring and tags only
  static constexpr size_t bytes = (STG || TMA) ? lead + barOff + 32 : ASY ? aS + (size_t)NS * NT * 4 : aF;
  static constexpr int warps = TY + 2;  // TY cell warps, the halo rows above and below, the sides
  static constexpr int threads = 32 * warps;
  static_assert(sizeof(Real) == 4, "the pipelined form holds FP32 arithmetic values in its ring");
  static_assert((ROWF * sizeof(PopT)) % 16 == 0 && (ROWH * sizeof(PopT)) % 16 == 0, "whole 16-byte units");
  static_assert(stF % 16 == 0 && stH % 16 == 0 && stM % 16 == 0 && stT % 16 == 0 && phiOff % 16 == 0,
                "bulk copy destinations are 16-byte aligned");
  static_assert(!TMA || (TY == TMA_ROWS && stF % 128 == 0 && stH % 128 == 0 && stM % 128 == 0 &&
                         (TY * MROW * sizeof(Real)) % 128 == 0 && stT % 128 == 0 && phiOff % 128 == 0 &&
                         (PSL * sizeof(Real)) % 128 == 0),
                "tensor copy destinations are 128-byte aligned; the maps' boxes are TMA_ROWS rows");
};

// ---------------------------------------------------------------- the tile
template <class PopT, int TY, int PF, bool WIDE, bool PACK = false>
__device__ __forceinline__ void fused_tile_pipe(const FusedArgs<PopT> &a, int bx, int by, int bz) {
  using POff = std::conditional_t<WIDE, long long, int>;
  using Real = typename Prec<PopT>::Real;
  using C = Codec<PopT>;
  using SM = PipeSmem<PopT, TY, PF>;
  constexpr bool STG = SM::STG, ASY = SM::ASY, TMA = SM::TMA, L2P = PF == PIPE_L2PF;
  using R = PipeRing<TY>;
  constexpr int CM = R::CM, CZ = R::CZ, CP = R::CP, CT = R::CT;
  using LD = CellLoad<PopT>;
  using CO = CellOut<PopT>;
  constexpr int RX = SM::RX, NC = SM::NC, TAGS = CT * NC, RING = R::TOTAL;
  constexpr int G27 = PopGroups<Q27>::G, G7 = PopGroups<Q7>::G;
  constexpr int BLK27 = PopGroups<Q27>::BLOCK, BLK7 = PopGroups<Q7>::BLOCK;
  constexpr int ROWF = SM::ROWF, ROWH = SM::ROWH, MROW = SM::MROW, TROW = SM::TROW, PROW = SM::PROW;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // the TMA form aligns its base up to 128 bytes (room for it is in SM::bytes)
  unsigned char *smem = smem_raw;
  if constexpr (SM::lead > 0) smem += (SM::lead - (smem_u32(smem_raw) & (SM::lead - 1))) & (SM::lead - 1);
  Real *ring = reinterpret_cast<Real *>(smem);
  uint8_t *stag = smem + SM::tagOff;                           // [3][NC]
  PopT *sF = reinterpret_cast<PopT *>(smem + SM::stF);         // [TY][ROWF]
  PopT *sH = reinterpret_cast<PopT *>(smem + SM::stH);         // [TY][ROWH]
  Real *sM = reinterpret_cast<Real *>(smem + SM::stM);         // [4][TY][MROW] rho ux uy uz
  uint8_t *sT = smem + SM::stT;                                // [TY][TROW]
  Real *sP = reinterpret_cast<Real *>(smem + SM::phiOff);      // [3][PSL]: TY + 2 rows of PROW
  const uint32_t bar = smem_u32(smem + SM::barOff);       // stage q landed (1 arrival + bytes)
  const uint32_t barE = smem_u32(smem + SM::barOff + 8);  // stage q read (one arrival per cell warp)
  int *abortF = reinterpret_cast<int *>(smem + SM::barOff + 16);

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
  const Real kappa = (Real)a.kappa, beta4 = (Real)a.beta4, rhoG = (Real)a.rhoG;
  const Real dRho = (Real)a.dRho, grav = (Real)a.gravity;
  const CollK<Real> K = coll_consts(a);

  const int tx = threadIdx.x, ty = threadIdx.y;
  const bool cellWarp = ty < TY, haloRows = ty == TY;
  const int x0 = bx * 32, y0 = by * TY;
  const int zb = 1 + bz * a.zchunk;
  const int ze = min(zb + a.zchunk, nz - 1);
  if (zb >= ze) return;
  const int x = x0 + tx, y = y0 + ty;
  const int own = (ty + 1) * RX + (tx + 1);  // tag-plane index of a cell warp's cell
  const int span = min(31, nx - 1 - x0);     // last column of the tile's rows
  const int r33 = ty * 33 + tx;

  // Lanes of the side warp: the left half (lanes 0..15) takes the left column
  // (lanes 0..TY-1 for rows 0..TY-1, then the corners at rows -1 and TY), the
  // right half (lanes 16..31) the right column the same way; each half
  // collides its side's directions (e_x = +1 on the left, -1 on the right).
  const bool sideRight = tx >= 16;
  const int sideLane = tx & 15;
  const bool sideAct = sideLane < TY + 2;
  const int sideLx = sideRight ? RX - 1 : 0;                                          // frame column
  const int sideLy = sideLane < TY ? sideLane + 1 : (sideLane == TY ? 0 : TY + 1);   // frame row
  const int sideSy = sideLane < TY ? 0 : (sideLane == TY ? 1 : -1);
  // the producer: lane 0 of cell warp 0 issues each stage as soon as every
  // cell warp has read the previous one (TMA: lane 0 of the halo-row warp,
  // after the barrier that follows those reads)
  const bool producer = (STG && ty == 0 && tx == 0) || (TMA && haloRows && tx == 0);

  // ---- halo loads (plain, into registers), as in fused_tile
  auto needs = [&](auto MODEc, auto SXc, auto SYc, auto KK, int sx, int sy,
                   bool active) __attribute__((always_inline)) -> bool {
    constexpr int MODE = decltype(MODEc)::value, SX = decltype(SXc)::value, SY = decltype(SYc)::value;
    constexpr int k = decltype(KK)::value;
    if constexpr (MODE == 0) return true;
    else if constexpr (MODE == 1) return active && halo_dir<SX, SY, k>();
    else return active && D27<k>::ex == SX && (sy == 0 || D27<k>::ey == sy);  // side: e_x fixed, e_y run time
  };
  auto load = [&](auto MODEc, auto SXc, auto SYc, int sx, int sy, bool active, int q, int gx_, int gy_,
                  LD &L) __attribute__((always_inline)) {
    constexpr int MODE = decltype(MODEc)::value, SX = decltype(SXc)::value, SY = decltype(SYc)::value;
    const bool inside = gx_ >= 0 && gx_ < nx && gy_ >= 0 && gy_ < ny && q >= 0 && q < nz;
    const int ci = inside ? q * nxny + gy_ * nx + gx_ : 0;
    const POff bF = (POff)(ci >> 3) * BLK27 + (ci & 7) * 4;
    const POff bH = (POff)(ci >> 3) * BLK7 + (ci & 7) * 4;
    // pad: element Q of the last group (ux for f, uy for h where they sit in
    // the pads), taken from that group's load where it is made
    auto groups = [&](auto QQ, auto NG, const PopT *src, POff base, long long lim, int code, PopT *dst,
                      PopT &pad) __attribute__((always_inline)) {
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
          if constexpr (4 * g + 3 == Q) pad = t[3];
        }
      });
    };
    PopT padF = PopT(), padH = PopT();
    groups(IC<Q27>{}, IC<G27>{}, Fc, bF, nF, 3, L.fv, padF);
    groups(IC<Q7>{}, IC<G7>{}, Hc, bH, nH, 4, L.hv, padH);
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
    if constexpr (UPAD && MODE == 0) {
      // a tile cell loads every group, the pads included
      L.ux = (Real)padF;
      L.uy = (Real)padH;
    } else if constexpr (UPAD) {
      L.ux = (Real)ldg_at(Fc, (long long)(ci >> 3) * BLK27 + (ci & 7) * 4 + pofs(27), nF, 6);
      L.uy = (Real)ldg_at(Hc, (long long)(ci >> 3) * BLK7 + (ci & 7) * 4 + pofs(7), nH, 6);
    } else {
      L.ux = ldg_at(uxC, ci, nCell, 6);
      L.uy = ldg_at(uyC, ci, nCell, 6);
    }
    L.uz = ldg_at(uzC, ci, nCell, 6);
    const bool inner = gx_ >= 1 && gx_ <= nx - 2 && gy_ >= 1 && gy_ <= ny - 2 && q >= 1 && q <= nz - 2;
    if (!inside || (!inner && tg == TAG_FLUID)) tg = TAG_WALL;
    L.tg = tg;
  };
  // the row warp's two cells (above and below the tile) share one load set's
  // worth of registers each; the side warp has one cell per lane
  auto halo_load = [&](int q, LD &L, LD &L2) __attribute__((always_inline)) {
    if (haloRows) {
      load(IC<1>{}, IC<0>{}, IC<1>{}, 0, 0, true, q, x, y0 - 1, L);
      load(IC<1>{}, IC<0>{}, IC<-1>{}, 0, 0, true, q, x, y0 + TY, L2);
    } else if (!sideRight) {
      load(IC<1>{}, IC<1>{}, IC<0>{}, 0, 0, sideAct, q, x0 - 1 + sideLx, y0 - 1 + sideLy, L);
    } else {
      load(IC<1>{}, IC<-1>{}, IC<0>{}, 0, 0, sideAct, q, x0 - 1 + sideLx, y0 - 1 + sideLy, L);
    }
  };

  // ---- the stage: bulk copies of plane q's tile rows (populations as whole
  // 8-cell blocks, rho / u as 16-byte aligned float runs, tags as 16-byte
  // aligned byte runs) and of plane q + 1's phi rows y0 - 1 .. y0 + TY, all
  // counted on one mbarrier.  Macro and tag arrays are allocated with a tail
  // pad, so the rounded-up end of the last row stays inside them.
  auto phi_row0 = [&](int P, int r) __attribute__((always_inline)) -> long long {
    // first element copied for phi row r (-1 .. TY) of plane P
    const long long c0 = ((long long)P * ny + (y0 + r)) * nx + x0 - 1;
    return c0 < 0 ? 0 : (c0 & ~3LL);
  };
  auto issue_phi = [&](int P, uint32_t &bytes, bool go) __attribute__((always_inline)) {
    if (P < 0 || P >= nz) return;
    for (int r = -1; r <= TY; r++) {
      const int yy = y0 + r;
      if (yy < 0 || yy >= ny) continue;
      const long long a0 = phi_row0(P, r);
      const long long c1 = ((long long)P * ny + yy) * nx + x0 + span + 1;
      const uint32_t cnt = (uint32_t)((c1 | 3) - a0 + 1);
      if (!lbm_ok(cnt <= PROW, 30, cnt) || !lbm_ok(a0 + cnt <= nCell + ARRAY_PAD, 40, a0)) continue;
      if (go)
        bulk_g2s(smem_u32(sP + (P % 3) * SM::PSL + (r + 1) * PROW), phiC + a0, cnt * sizeof(Real), bar);
      else
        bytes += cnt * sizeof(Real);
    }
  };
  auto issue_rows = [&](int q, uint32_t &bytes, bool go) __attribute__((always_inline)) {
    for (int r = 0; r < TY; r++) {
      const int yy = y0 + r;
      if (yy >= ny) break;
      const long long row0 = ((long long)q * ny + yy) * nx + x0;
      const long long b0 = row0 >> 3;
      const uint32_t nb = (uint32_t)(((row0 + span) >> 3) - b0 + 1);
      const long long m0 = row0 & ~3LL, t0 = row0 & ~15LL;
      const uint32_t mcnt = (uint32_t)(((row0 + span) | 3) - m0 + 1);
      const uint32_t tcnt = (uint32_t)(((row0 + span) | 15) - t0 + 1);
      const bool ok = lbm_ok(nb <= (uint32_t)SM::SB, 31, nb) && lbm_ok((b0 + nb) * BLK27 <= nF, 32, b0) &&
                      lbm_ok(mcnt <= (uint32_t)MROW, 33, mcnt) && lbm_ok(tcnt <= (uint32_t)TROW, 34, tcnt) &&
                      lbm_ok(m0 + mcnt <= nCell + ARRAY_PAD, 41, m0) && lbm_ok(t0 + tcnt <= nCell + ARRAY_PAD, 42, t0);
      if (!ok) continue;
      if (go) {
        bulk_g2s(smem_u32(sF + r * ROWF), Fc + b0 * BLK27, nb * BLK27 * sizeof(PopT), bar);
        bulk_g2s(smem_u32(sH + r * ROWH), Hc + b0 * BLK7, nb * BLK7 * sizeof(PopT), bar);
        bulk_g2s(smem_u32(sM + (0 * TY + r) * MROW), rhoC + m0, mcnt * sizeof(Real), bar);
        bulk_g2s(smem_u32(sM + (1 * TY + r) * MROW), uxC + m0, mcnt * sizeof(Real), bar);
        bulk_g2s(smem_u32(sM + (2 * TY + r) * MROW), uyC + m0, mcnt * sizeof(Real), bar);
        bulk_g2s(smem_u32(sM + (3 * TY + r) * MROW), uzC + m0, mcnt * sizeof(Real), bar);
        bulk_g2s(smem_u32(sT + r * TROW), tagA + t0, tcnt, bar);
      } else {
        bytes += nb * (BLK27 + BLK7) * sizeof(PopT) + 4 * mcnt * sizeof(Real) + tcnt;
      }
    }
  };
  // stage(q): rows of plane q and phi of plane q + 1 (prologue: also phi of
  // planes q - 1 and q)
  auto issue = [&](int q, bool prologue) __attribute__((always_inline)) {
    uint32_t bytes = 0;
    issue_rows(q, bytes, false);
    issue_phi(q + 1, bytes, false);
    if (prologue) {
      issue_phi(q - 1, bytes, false);
      issue_phi(q, bytes, false);
    }
    mbar_expect(bar, bytes);
    issue_rows(q, bytes, true);
    issue_phi(q + 1, bytes, true);
    if (prologue) {
      issue_phi(q - 1, bytes, true);
      issue_phi(q, bytes, true);
    }
  };

  // TMA stage(q): rows of plane q and phi of plane q + 1 (prologue: also phi
  // of planes q - 1 and q), one box per array.  Boxes reaching outside the
  // grid (the right-hand tile's last blocks, rows past ny, planes -1 and nz,
  // columns x0 - 4 .. x0 - 1 of the first tile) bring zeros, which only cells
  // outside the grid and boundary cells (walls) read.
  auto issue_tma = [&](int q, bool prologue) __attribute__((always_inline)) {
    const StageMaps *m = a.maps;
    mbar_expect(bar, SM::tmaRows + (prologue ? 3u : 1u) * SM::tmaPhi);
    tma_g2s_4d(smem_u32(sF), &m->f[cur], 0, x0 >> 3, y0, q, bar);
    tma_g2s_4d(smem_u32(sH), &m->h[cur], 0, x0 >> 3, y0, q, bar);
    tma_g2s_3d(smem_u32(sM), &m->rho[cur], x0, y0, q, bar);
    if constexpr (!UPAD) {
      tma_g2s_3d(smem_u32(sM + 1 * TY * MROW), &m->ux[cur], x0, y0, q, bar);
      tma_g2s_3d(smem_u32(sM + 2 * TY * MROW), &m->uy[cur], x0, y0, q, bar);
    }
    tma_g2s_3d(smem_u32(sM + 3 * TY * MROW), &m->uz[cur], x0, y0, q, bar);
    tma_g2s_3d(smem_u32(sT), &m->tag, x0, y0, q, bar);
    auto phi = [&](int P) __attribute__((always_inline)) {
      const int slot = P - 3 * (int)((unsigned)(P + 3) / 3u) + 3;  // P mod 3 for P >= -1
      tma_g2s_3d(smem_u32(sP + slot * SM::PSL), &m->phi[cur], x0 - 4, y0 - 1, P, bar);
    };
    phi(q + 1);
    if (prologue) {
      phi(q - 1);
      phi(q);
    }
  };

  // L2 prefetch of plane P's tile rows (and phi of plane P + 1, rows y0 - 1 ..
  // y0 + TY), the boxes and coordinates of issue_tma
  auto prefetch_l2 = [&](int P) __attribute__((always_inline)) {
    const StageMaps *m = a.maps;
    tma_l2_4d(&m->f[cur], 0, x0 >> 3, y0, P);
    tma_l2_4d(&m->h[cur], 0, x0 >> 3, y0, P);
    tma_l2_3d(&m->rho[cur], x0, y0, P);
    if constexpr (!UPAD) {
      tma_l2_3d(&m->ux[cur], x0, y0, P);
      tma_l2_3d(&m->uy[cur], x0, y0, P);
    }
    tma_l2_3d(&m->uz[cur], x0, y0, P);
    tma_l2_3d(&m->tag, x0, y0, P);
    tma_l2_3d(&m->phi[cur], x0 - 4, y0 - 1, P + 1);
  };

  // a cell warp's cell of plane q from the stage.  Positions inside the staged
  // rows follow from the rows' first flat indices modulo 16, computed in
  // 32-bit arithmetic (2^32 is a multiple of 16).
  auto stage_load = [&](int q, LD &L) __attribute__((always_inline)) {
    const bool inside = x < nx && y < ny;
    const int t = inside ? tx : 0;
    const uint32_t rowlo = ((uint32_t)q * (uint32_t)ny + (uint32_t)y) * (uint32_t)nx + (uint32_t)x0;
    const int b = (int)(rowlo & 7u) + t;  // cell position from the start of the row's first block
    const int off = b >> 3, e = b & 7;
    const PopT *f = sF + ty * ROWF, *h = sH + ty * ROWH;
    static_for<0, G27>([&](auto GG) {
      constexpr int g = decltype(GG)::value;
      PopT tv[4];
      ld4_shared(f + sm_at((off * G27 + g) * 32 + e * 4, ROWF - 3, 35), tv);
      static_for<4 * g, (4 * g + 4 < Q27 ? 4 * g + 4 : Q27)>([&](auto KK) {
        constexpr int k = decltype(KK)::value;
        L.fv[k] = tv[k & 3];
      });
      if constexpr (g < G7) {
        ld4_shared(h + sm_at((off * G7 + g) * 32 + e * 4, ROWH - 3, 36), tv);
        static_for<4 * g, (4 * g + 4 < Q7 ? 4 * g + 4 : Q7)>([&](auto KK) {
          constexpr int k = decltype(KK)::value;
          L.hv[k] = tv[k & 3];
        });
      }
    });
    const int mi = sm_at((int)(rowlo & 3u) + t, MROW, 37);
    L.sumF = sM[(0 * TY + ty) * MROW + mi];
    if constexpr (UPAD) {  // in the pads of the staged rows' last groups
      L.ux = (Real)f[sm_at((off * G27 + 6) * 32 + e * 4 + 3, ROWF, 35)];
      L.uy = (Real)h[sm_at((off * G7 + 1) * 32 + e * 4 + 3, ROWH, 36)];
    } else {
      L.ux = sM[(1 * TY + ty) * MROW + mi];
      L.uy = sM[(2 * TY + ty) * MROW + mi];
    }
    L.uz = sM[(3 * TY + ty) * MROW + mi];
    uint8_t tg = sT[ty * TROW + sm_at((int)(rowlo & 15u) + t, TROW, 38)];
    // phi stencil: staged rows ty (y - 1), ty + 1 (y), ty + 2 (y + 1) of plane
    // q and row ty + 1 of planes q - 1 and q + 1.  A staged phi row starts at
    // the 16-byte unit holding cell x0 - 1; indices are clamped into the row
    // (only boundary cells, which are walls, reach a clamp).
    auto pat = [&](int P, int rr, int dx) __attribute__((always_inline)) -> Real {
      const uint32_t c0 = ((uint32_t)P * (uint32_t)ny + (uint32_t)(y0 + rr - 1)) * (uint32_t)nx + (uint32_t)x0 - 1u;
      int i = t + 1 + dx + (int)(c0 & 3u);
      i = i < 0 ? 0 : (i >= PROW ? PROW - 1 : i);
      const int slot = P - 3 * (int)((unsigned)(P + 3) / 3u) + 3;  // P mod 3 for P >= -1
      return sP[slot * SM::PSL + rr * PROW + sm_at(i, PROW, 39)];
    };
    L.p = pat(q, ty + 1, 0);
    L.pxp = pat(q, ty + 1, 1);
    L.pxm = pat(q, ty + 1, -1);
    L.pyp = pat(q, ty + 2, 0);
    L.pym = pat(q, ty, 0);
    L.pzp = pat(q + 1, ty + 1, 0);
    L.pzm = pat(q - 1, ty + 1, 0);
    const bool inner = x >= 1 && x <= nx - 2 && y >= 1 && y <= ny - 2 && q >= 1 && q <= nz - 2;
    if (!inside || (!inner && tg == TAG_FLUID)) tg = TAG_WALL;
    L.tg = tg;
  };

  // ---- emit: collided values and tag of a cell into the ring (local cell lx, ly)
  auto emit = [&](auto MODEc, auto SXc, auto SYc, int sx, int sy, bool active, int q, int lx, int ly,
                  const CO &o) __attribute__((always_inline)) {
    constexpr int MODE = decltype(MODEc)::value, SX = decltype(SXc)::value, SY = decltype(SYc)::value;
    const int qM = ring_copy<CM>(q), qZ = ring_copy<CZ>(q), qP = ring_copy<CP>(q);
    const int cM = R::FM + qM * R::grp(27, -1), cZ = R::FZ + qZ * R::grp(27, 0);
    const int cP = R::FP + qP * R::grp(27, 1);
    const int hM = R::HM + qM * R::grp(7, -1), hZ = R::HZ + qZ * R::grp(7, 0);
    const int hP = R::HP + qP * R::grp(7, 1);
    const int lc = (ly + 1) * RX + (lx + 1);
    if (MODE != 2 || active) stag[sm_at(ring_copy<CT>(q) * NC + lc, TAGS, 2)] = (MODE == 1 && SY < 0) ? o.tg2 : o.tg;
    static_for<0, Q27>([&](auto KK) {
      constexpr int k = decltype(KK)::value;
      constexpr int ez = kDir[k][2];
      if constexpr (MODE == 0 || (MODE == 1 && halo_dir<SX, SY, k>()) || (MODE == 2 && kDir[k][0] == SX)) {
        const bool nd = needs(MODEc, SXc, SYc, KK, sx, sy, active);
        const int base = ez < 0 ? cM : (ez == 0 ? cZ : cP);
        int idx;
        if constexpr (MODE == 0) {
          idx = base + r33 + R::at(27, k, 0, 0);
        } else {
          idx = base + R::off(27, k) + (ly - R::RY0(k)) * R::W(k) + (lx - R::CX0(k));
        }
        if (nd) ring[sm_at(idx, RING, 7)] = o.f[k];
        if constexpr (k < Q7) {
          const int hb = ez < 0 ? hM : (ez == 0 ? hZ : hP);
          int hidx;
          if constexpr (MODE == 0) hidx = hb + r33 + R::at(7, k, 0, 0);
          else hidx = hb + R::off(7, k) + (ly - R::RY0(k)) * R::W(k) + (lx - R::CX0(k));
          if (nd) ring[sm_at(hidx, RING, 8)] = o.h[k];
        }
      }
    });
  };

  // ---- the async form: a cell warp's cell of plane q into this thread's own
  // slots (every group of f and h, phi and its six neighbours, rho, u) by
  // per-thread asynchronous copies from the same clamped addresses the plain
  // load uses; the tag (one byte, no copy size that small) by a plain load
  // into a register that is held until plane q is collided
  constexpr int NT = SM::NT, GB = SM::GB;
  PopT *aF = reinterpret_cast<PopT *>(smem + SM::aF);  // [G27][NT] groups
  PopT *aH = reinterpret_cast<PopT *>(smem + SM::aH);  // [G7][NT] groups
  Real *aS = reinterpret_cast<Real *>(smem + SM::aS);  // [11][NT] words
  const int lin = ty * 32 + tx;
  auto async_issue = [&](int q, uint8_t &tgq) __attribute__((always_inline)) {
    const bool inside = x < nx && y < ny && q >= 0 && q < nz;
    const int ci = inside ? q * nxny + y * nx + x : 0;
    const POff bF = (POff)(ci >> 3) * BLK27 + (ci & 7) * 4;
    const POff bH = (POff)(ci >> 3) * BLK7 + (ci & 7) * 4;
    static_for<0, G27>([&](auto GG) {
      constexpr int g = decltype(GG)::value;
      const long long e = (long long)bF + 32 * g;
      if (lbm_ok(e >= 0 && e + 3 < nF, 3, e)) cp_async<GB>(smem_u32(aF + (g * NT + lin) * 4), Fc + e);
    });
    static_for<0, G7>([&](auto GG) {
      constexpr int g = decltype(GG)::value;
      const long long e = (long long)bH + 32 * g;
      if (lbm_ok(e >= 0 && e + 3 < nH, 4, e)) cp_async<GB>(smem_u32(aH + (g * NT + lin) * 4), Hc + e);
    });
    const int last = (int)nCell - 1;
    const int src[SM::NS] = {ci, min(ci + 1, last), max(ci - 1, 0), min(ci + nx, last), max(ci - nx, 0),
                             min(ci + nxny, last), max(ci - nxny, 0), ci, ci, ci, ci};
    const Real *arr[SM::NS] = {phiC, phiC, phiC, phiC, phiC, phiC, phiC, rhoC, uxC, uyC, uzC};
#pragma unroll
    for (int j = 0; j < SM::NS; j++) {
      if (UPAD && (j == 8 || j == 9)) continue;  // ux, uy arrive in the pads of the group slots
      if (lbm_ok(src[j] >= 0 && src[j] < nCell, j < 7 ? 5 : 6, src[j]))
        cp_async<4>(smem_u32(aS + j * NT + lin), arr[j] + src[j]);
    }
    cp_async_commit();
    tgq = ldg_at(tagA, ci, nCell, 1);
  };
  auto async_load = [&](int q, uint8_t tgq, LD &L) __attribute__((always_inline)) {
    cp_async_wait_all();
    static_for<0, G27>([&](auto GG) {
      constexpr int g = decltype(GG)::value;
      PopT tv[4];
      ld4_shared(aF + (g * NT + lin) * 4, tv);
      static_for<4 * g, (4 * g + 4 < Q27 ? 4 * g + 4 : Q27)>([&](auto KK) {
        constexpr int k = decltype(KK)::value;
        L.fv[k] = tv[k & 3];
      });
      if constexpr (g < G7) {
        ld4_shared(aH + (g * NT + lin) * 4, tv);
        static_for<4 * g, (4 * g + 4 < Q7 ? 4 * g + 4 : Q7)>([&](auto KK) {
          constexpr int k = decltype(KK)::value;
          L.hv[k] = tv[k & 3];
        });
      }
    });
    L.p = aS[0 * NT + lin];
    L.pxp = aS[1 * NT + lin];
    L.pxm = aS[2 * NT + lin];
    L.pyp = aS[3 * NT + lin];
    L.pym = aS[4 * NT + lin];
    L.pzp = aS[5 * NT + lin];
    L.pzm = aS[6 * NT + lin];
    L.sumF = aS[7 * NT + lin];
    if constexpr (UPAD) {
      L.ux = (Real)aF[(6 * NT + lin) * 4 + 3];
      L.uy = (Real)aH[(1 * NT + lin) * 4 + 3];
    } else {
      L.ux = aS[8 * NT + lin];
      L.uy = aS[9 * NT + lin];
    }
    L.uz = aS[10 * NT + lin];
    uint8_t tg = tgq;
    const bool inside = x < nx && y < ny;
    const bool inner = x >= 1 && x <= nx - 2 && y >= 1 && y <= ny - 2 && q >= 1 && q <= nz - 2;
    if (!inside || (!inner && tg == TAG_FLUID)) tg = TAG_WALL;
    L.tg = tg;
  };

  Real gxC = 0, gyC = 0, gzC = 0, lapC = 0, phC = 0;
  Real gxN = 0, gyN = 0, gzN = 0, lapN = 0, phN = 0;
  const bool colActive = cellWarp && x >= 1 && x <= nx - 2 && y >= 1 && y <= ny - 2;

  if (producer) {
    mbar_init(bar);
    if constexpr (STG) mbar_init_count(barE, TY);
    mbar_init_fence();
    if constexpr (TMA) fence_proxy_async();  // the initialised mbarrier, seen by the tensor copies
  }
  if ((STG || TMA) && threadIdx.x == 0 && threadIdx.y == 0) *abortF = 0;
  __syncthreads();
  if (producer && !a.withhold) {
    if constexpr (TMA) issue_tma(zb - 1, true);
    else issue(zb - 1, true);
  }
  uint32_t parity = 0;
  uint8_t tgNext = 0;
  if constexpr (ASY) {
    if (cellWarp) async_issue(zb - 1, tgNext);
  }

  int q = zb - 1;
  for (; q <= ze; q++) {
    CO o;
    if (cellWarp) {
      LD L;
      if constexpr (STG) {
        if (!mbar_wait(bar, parity)) {
          record_stage_timeout(q);
          if (a.status) atomicOr(a.status, 1);
          *abortF = 1;
        }
        stage_load(q, L);
        __syncwarp();
        if (tx == 0) mbar_arrive(barE);
        if (producer) {
          // every cell warp has its plane-q values in registers: the stage and
          // the phi slot of plane q - 1 are free for stage q + 1, which now
          // lands while plane q is collided and plane q - 1 pulled.  A wait
          // that ran out (set before the arrivals) stops the issuing.
          if (mbar_wait(barE, parity) && q < ze && !*abortF) issue(q + 1, false);
        }
      } else if constexpr (TMA) {
        if (!mbar_wait(bar, parity)) {
          record_stage_timeout(q);
          if (a.status) atomicOr(a.status, 1);
          *abortF = 1;
        }
        stage_load(q, L);
      } else if constexpr (ASY) {
        async_load(q, tgNext, L);
      } else {
        load(IC<0>{}, IC<0>{}, IC<0>{}, 0, 0, true, q, x, y, L);
      }
      collide_cell<PopT, 0, 0, 0>(K, L, o, gxN, gyN, gzN, lapN, phN);
    } else {
      // the halo warps load after the barrier that ends the previous plane,
      // while the cell warps pull it: their latency is off the critical path
      Real d0, d1, d2, d3, d4;
      LD Lh, Lh2;
      halo_load(q, Lh, Lh2);
      if (haloRows) {
        collide_cell<PopT, 1, 0, 1>(K, Lh, o, d0, d1, d2, d3, d4);
        collide_cell<PopT, 1, 0, -1>(K, Lh2, o, d0, d1, d2, d3, d4);
      } else if (!sideRight) {
        collide_cell<PopT, 1, 1, 0>(K, Lh, o, d0, d1, d2, d3, d4);
      } else {
        collide_cell<PopT, 1, -1, 0>(K, Lh, o, d0, d1, d2, d3, d4);
      }
    }
    parity ^= 1u;
    // every warp has pulled plane q - 2 and the cell warps have read the stage
    __syncthreads();
    if constexpr (L2P) {
      // plane q + 2 (q + 3) into L2 (the cell warps load plane q + 1 next,
      // so this has at least a plane and a half to land); planes past the
      // chunk's last are not needed
      constexpr int AH = l2pf_ahead<PopT>();
      if (haloRows && tx == 0 && a.maps && q + AH <= ze) prefetch_l2(q + AH);
    }
    if constexpr (TMA) {
      // stage q + 1 into the buffers of stage q, which every cell warp read
      // before the barrier above; it lands while plane q is emitted and plane
      // q - 1 pulled.  A wait that ran out (set before the barrier) stops it.
      if (producer && q < ze && !*abortF) {
        fence_proxy_async();
        issue_tma(q + 1, false);
      }
    }
    if (cellWarp) {
      emit(IC<0>{}, IC<0>{}, IC<0>{}, 0, 0, true, q, tx, ty, o);
      // the slots of plane q were read before the barrier above: plane q + 1
      // now lands while plane q - 1 is pulled
      if constexpr (ASY) {
        if (q < ze) async_issue(q + 1, tgNext);
      }
    } else if (haloRows) {
      emit(IC<1>{}, IC<0>{}, IC<1>{}, 0, 0, true, q, tx, -1, o);
      emit(IC<1>{}, IC<0>{}, IC<-1>{}, 0, 0, true, q, tx, TY, o);
    } else if (!sideRight) {
      emit(IC<2>{}, IC<1>{}, IC<0>{}, 1, sideSy, sideAct, q, sideLx - 1, sideLy - 1, o);
    } else {
      emit(IC<2>{}, IC<-1>{}, IC<0>{}, -1, sideSy, sideAct, q, sideLx - 1, sideLy - 1, o);
    }
    __syncthreads();
    if constexpr (STG || TMA) {
      if (*abortF) break;
    }

    // pull plane z = q - 1 (nothing while z < zb)
    const int z = q - 1;
    const int sC = ring_copy<CT>(z);
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
      // ring copies: group e_z sources come from plane z - e_z; the cell's own
      // (bounce-back) values are in plane z
      const int zMs = ring_copy<CM>(z + 1), zMo = ring_copy<CM>(z), zZ = ring_copy<CZ>(z);
      const int zPs = ring_copy<CP>(z - 1), zPo = ring_copy<CP>(z);
      const int sFM = R::FM + zMs * R::grp(27, -1), sFZ = R::FZ + zZ * R::grp(27, 0);
      const int sFP = R::FP + zPs * R::grp(27, 1);
      const int oFM = R::FM + zMo * R::grp(27, -1), oFP = R::FP + zPo * R::grp(27, 1);
      const int sHM = R::HM + zMs * R::grp(7, -1), sHZ = R::HZ + zZ * R::grp(7, 0);
      const int sHP = R::HP + zPs * R::grp(7, 1);
      const int oHM = R::HM + zMo * R::grp(7, -1), oHP = R::HP + zPo * R::grp(7, 1);
      const int tbM = ring_copy<CT>(z + 1) * NC + own, tbZ = sC * NC + own, tbP = ring_copy<CT>(z - 1) * NC + own;
      const Real rhoPhOld = rfma(phC, dRho, rhoG);
      Real rhoA = 0, mx = 0, my = 0, mz = 0, hsum = 0;
      Real hn[Q7];
      Real val4[4], ref4[4];
      PopT enc4[4], lastF[4];
      uint32_t orTags = 0;
      static_for<0, Q27>([&](auto KK) {
        constexpr int k = decltype(KK)::value;
        using D = D27<k>;
        constexpr int ex = D::ex, ey = D::ey, ez = D::ez, o = D::opp;
        constexpr int oz = D27<o>::ez;
        constexpr int so = -ey * RX - ex;
        const int tb = ez < 0 ? tbM : (ez == 0 ? tbZ : tbP);
        const int sbF = ez < 0 ? sFM : (ez == 0 ? sFZ : sFP);
        const int obF = oz < 0 ? oFM : (oz == 0 ? sFZ : oFP);
        const uint8_t ts = stag[sm_at(tb + so, TAGS, 13)];
        const bool fl = ts == TAG_FLUID;
        // source (tx - ex, ty - ey) in direction k's array; own cell in o's.
        // Both are read and the value selected, so each load keeps its
        // compile-time offset and no address is selected per direction.
#ifdef LBM_CHECKED
        const int si = sbF + r33 + R::at(27, k, -ex, -ey);
        const int oi = obF + r33 + R::at(27, o, 0, 0);
        const Real fk = ring[sm_at(fl ? si : oi, RING, 14)];
#else
        const Real fS = ring[sbF + r33 + R::at(27, k, -ex, -ey)];
        const Real fO = ring[obF + r33 + R::at(27, o, 0, 0)];
        const Real fk = fl ? fS : fO;
#endif
        orTags |= ts;
        val4[k & 3] = fk;
        ref4[k & 3] = (Real)D::w;
        if constexpr ((k & 3) == 3 || k == Q27 - 1) {
          if constexpr (k == Q27 - 1) val4[3] = ref4[3] = 0;  // pad of the last group: encodes to +0
          C::enc4(val4, ref4, enc4);
          if constexpr (UPAD && k == Q27 - 1) {
            // the last group waits for ux, its pad (stored at once below
            // where SOLID links rewrite its elements)
            lastF[0] = enc4[0], lastF[1] = enc4[1], lastF[2] = enc4[2], lastF[3] = enc4[3];
          } else {
            st4_at(Fn, bF + pofs(k & ~3), nF, 15, enc4);
          }
        }
        rhoA += fk;
        if constexpr (ex != 0) mx += (Real)ex * fk;
        if constexpr (ey != 0) my += (Real)ey * fk;
        if constexpr (ez != 0) mz += (Real)ez * fk;
        if constexpr (k < Q7) {
          const int sbH = ez < 0 ? sHM : (ez == 0 ? sHZ : sHP);
          const int obH = oz < 0 ? oHM : (oz == 0 ? sHZ : oHP);
#ifdef LBM_CHECKED
          const int shi = sbH + r33 + R::at(7, k, -ex, -ey);
          const int ohi = obH + r33 + R::at(7, o, 0, 0);
          const Real hk = ring[sm_at(fl ? shi : ohi, RING, 16)];
#else
          const Real hS = ring[sbH + r33 + R::at(7, k, -ex, -ey)];
          const Real hO = ring[obH + r33 + R::at(7, o, 0, 0)];
          const Real hk = fl ? hS : hO;
#endif
          hn[k] = hk;
          hsum += hk;
        }
      });
      // Links to SOLID sources (rare): Ladd moving-wall term and the FP64
      // momentum exchange (src/sim.js:517-536), directions from a bit mask.
      static_assert(TAG_FLUID == 0 && (TAG_SOLID & TAG_WALL) == 0, "tag bits");
      if (orTags & TAG_SOLID) {
        if constexpr (UPAD) st4_at(Fn, bF + pofs(Q27 - 3), nF, 15, lastF);  // before the links rewrite it
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
          // own value of the opposite direction o at (tx, ty) in plane z
          int oi = oz < 0 ? oFM : (oz == 0 ? sFZ : oFP);
          static_for<1, Q27>([&](auto KK) {
            constexpr int kk = decltype(KK)::value;
            if (kk == o) oi += r33 + R::at(27, kk, 0, 0);
          });
          const Real fopp = ring[sm_at(oi, RING, 19)];
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
      // h, the last group's pad holding uy where u sits in the pads (the
      // FP32 / FP64 codec stores it unchanged), +0 otherwise
      static_for<0, Q7>([&](auto KK) {
        constexpr int k = decltype(KK)::value;
        val4[k & 3] = hn[k];
        ref4[k & 3] = (Real)D7<k>::w * p;
        if constexpr ((k & 3) == 3 || k == Q7 - 1) {
          if constexpr (k == Q7 - 1) {
            val4[3] = UPAD ? uyn : (Real)0;
            ref4[3] = 0;
          }
          C::enc4(val4, ref4, enc4);
          st4_at(Hn, bH + pofs(k & ~3), nH, 17, enc4);
        }
      });
      st_at(s.rho[nxt], i, nCell, 18, rhoN);
      st_at(s.phi[nxt], i, nCell, 18, p);
      if constexpr (UPAD) {
        // f's last group with ux in its pad (where SOLID links were written,
        // the group went out above and only the pad remains)
        if (orTags & TAG_SOLID) {
          st_at(Fn, bF + pofs(27), nF, 18, (PopT)uxn);
        } else {
          lastF[3] = (PopT)uxn;
          st4_at(Fn, bF + pofs(Q27 - 3), nF, 15, lastF);
        }
      } else {
        st_at(s.ux[nxt], i, nCell, 18, uxn);
        st_at(s.uy[nxt], i, nCell, 18, uyn);
      }
      st_at(s.uz[nxt], i, nCell, 18, uzn);
      if (PACK && lbm_ok(i < nCell, 50, i)) pack_rg8(a.pack, i, p, false);
    } else if (PACK && cellWarp && x < nx && y < ny && z >= zb) {
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

  // Stopped early (a wait ran out): the copy of stage q was issued (unless
  // withheld) and may still be in flight; let it land (bounded) before the
  // shared memory is released.  Normal exit: every issued copy was waited for.
  if constexpr (STG || TMA) {
    if (q <= ze && producer && !(a.withhold && q == zb - 1)) mbar_wait(bar, parity ^ 1u);
    __syncthreads();
    if (producer) {
      mbar_inval(bar);
      if constexpr (STG) mbar_inval(barE);
    }
  }
}

// CTAs per SM the register budget is sized for: 4 rows fit three CTAs per SM
// in shared memory, 6 rows two
template <int TY, int PF>
struct PipeOcc {
  static constexpr int blocks = TY <= 4 ? 3 : 2;
};

template <class PopT, int TY, int PF, bool WIDE, bool PACK = false>
__global__ void __launch_bounds__(32 * (TY + 2), PipeOcc<TY, PF>::blocks)
    k_fused_pipe(const __grid_constant__ FusedArgs<PopT> a) {
  fused_tile_pipe<PopT, TY, PF, WIDE, PACK>(a, blockIdx.x, blockIdx.y, blockIdx.z);
}

// Many scenes in one persistent launch (as k_fused_batch)
template <class PopT, int TY, int PF, bool WIDE>
__global__ void __launch_bounds__(32 * (TY + 2), PipeOcc<TY, PF>::blocks)
    k_fused_pipe_batch(const FusedArgs<PopT> *__restrict__ args, const int *__restrict__ tileStart,
                       const int3 *__restrict__ tileGrid, int nscenes) {
  const int total = tileStart[nscenes];
  for (int w = blockIdx.x; w < total; w += gridDim.x) {
    int lo = 0, hi = nscenes - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (tileStart[mid] <= w) lo = mid;
      else hi = mid - 1;
    }
    const int3 g = tileGrid[lo];
    const int t = w - tileStart[lo];
    const int bx = t % g.x, by = (t / g.x) % g.y, bz = t / (g.x * g.y);
    __shared__ FusedArgs<PopT> sa;
    constexpr int WORDS = sizeof(FusedArgs<PopT>) / 4;
    const int lin = threadIdx.y * blockDim.x + threadIdx.x;
    if (lin < WORDS)
      reinterpret_cast<uint32_t *>(&sa)[lin] = reinterpret_cast<const uint32_t *>(args + lo)[lin];
    __syncthreads();
    fused_tile_pipe<PopT, TY, PF, WIDE>(sa, bx, by, bz);
    __syncthreads();
  }
}

}  // namespace lbm
