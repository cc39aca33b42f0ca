// Typed kernel launchers: Ops<PopT> implements OpsBase for one population
// storage type.  Included once per storage type by lbm_inst_*.cu.
#pragma once

#include <cudaTypedefs.h>  // the driver's tensor-map encoder type
#include <string.h>

#include <algorithm>

#include "lbm_fused_pipe.cuh"
#include "lbm_kernels.cuh"
#include "lbm_sphere.cuh"
#include "lbm_state.h"

namespace lbm {

static_assert(sizeof(TensorMap) == sizeof(CUtensorMap) && alignof(TensorMap) == alignof(CUtensorMap),
              "TensorMap holds one CUtensorMap");

// The driver's tensor-map encoder, looked up once through the runtime (no
// link against the driver library); null where the driver lacks it.
inline PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = []() -> PFN_cuTensorMapEncodeTiled_v12000 {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// ---------------------------------------------------------------- transfers
template <class PopT>
__global__ void k_aos_to_soa(Scene<PopT, typename Prec<PopT>::Real> s, int isH, int half, int cur,
                             const float *aos, long long c0, long long cells) {
  using Real = typename Prec<PopT>::Real;
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= cells) return;
  long long i = c0 + c;
  const int Q = isH ? Q7 : Q27;
  for (int hf = 0; hf < 2; hf++) {
    int dst = hf == 0 ? cur : 1 - cur;
    if (half == 1 && dst != cur) continue;
    if (half == 2 && dst == cur) continue;
    PopT *P = isH ? s.H[dst] : s.F[dst];
    for (int k = 0; k < Q; k++) {
      Real v = (Real)aos[c * Q + k];
      Real ref = isH ? (Real)w7_of(k) * s.phi[dst][i] : (Real)w27_of(k);
      P[isH ? pidx<7>(k, i) : pidx<27>(k, i)] = Codec<PopT>::enc(v, ref);
    }
  }
}

template <class PopT, class OutT>
__global__ void k_soa_to_aos(Scene<PopT, typename Prec<PopT>::Real> s, int isH, int src, OutT *aos,
                             long long c0, long long cells) {
  using Real = typename Prec<PopT>::Real;
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= cells) return;
  long long i = c0 + c;
  const int Q = isH ? Q7 : Q27;
  const PopT *P = isH ? s.H[src] : s.F[src];
  for (int k = 0; k < Q; k++) {
    Real ref = isH ? (Real)w7_of(k) * s.phi[src][i] : (Real)w27_of(k);
    aos[c * Q + k] = (OutT)Codec<PopT>::dec(P[isH ? pidx<7>(k, i) : pidx<27>(k, i)], ref);
  }
}

template <class PopT>
__global__ void k_reencode_h(Scene<PopT, typename Prec<PopT>::Real> s, int half,
                             const typename Prec<PopT>::Real *oldPhi) {
  using Real = typename Prec<PopT>::Real;
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= s.n) return;
  Real po = oldPhi[i], pn = s.phi[half][i];
  for (int k = 0; k < Q7; k++) {
    Real w = (Real)w7_of(k);
    Real v = Codec<PopT>::dec(s.H[half][pidx<7>(k, i)], w * po);
    s.H[half][pidx<7>(k, i)] = Codec<PopT>::enc(v, w * pn);
  }
}

// The device-resident loop's RigidSphere.step(1.0, gravity), one thread per
// sphere: the momentum-exchange and dead-cell impulses of the step are added
// first, as RigidSphere.applyImpulseAtCell would have.
__device__ __forceinline__ void sphere_step_body(lbm_sphere *sph, int nsph, double gravity, const double *fluid,
                                                 const double *dead, int nx, int ny, int nz) {
  int b = threadIdx.x;
  if (b >= nsph) return;
  lbm_sphere s = sph[b];
  double *F[6] = {&s.Fx, &s.Fy, &s.Fz, &s.Tx, &s.Ty, &s.Tz};
  for (int j = 0; j < 6; j++) {
    if (fluid) *F[j] = __dadd_rn(*F[j], fluid[6 * b + j]);
    if (dead) *F[j] = __dadd_rn(*F[j], dead[6 * b + j]);
  }
  sphere_step_fp64(s, 1.0, gravity, nx, ny, nz);
  sph[b] = s;
}
static __global__ void k_sphere_step(lbm_sphere *sph, int nsph, double gravity, const double *fluid,
                                     const double *dead, int nx, int ny, int nz) {
  if (blockIdx.x != 0) return;
  sphere_step_body(sph, nsph, gravity, fluid, dead, nx, ny, nz);
}

// ---------------------------------------------------------------- batched sparse kernels
// A batch runs every scene's sparse kernels of a step (plan, retag, fresh /
// dead compaction, fresh fill; after the shared fused launch the impulse
// reduction, the dead-cell impulses and the sphere step) as one launch per
// kind: grid row (or plane) s runs scene s's kernel body on scene s's
// arguments, so a step of n scenes costs 9 launches instead of 9 n.
// ux (comp 0) or uy (comp 1) of one half between a plain array and the
// place the scene keeps it (Scene::ux_at / set_ux), for the field transfers
template <class PopT>
__global__ void k_u_array(Scene<PopT, typename Prec<PopT>::Real> s, int comp, int half,
                          typename Prec<PopT>::Real *arr, int toScene) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= s.n) return;
  if (toScene) {
    if (comp == 0) s.set_ux(half, i, arr[i]);
    else s.set_uy(half, i, arr[i]);
  } else {
    arr[i] = comp == 0 ? s.ux_at(half, i) : s.uy_at(half, i);
  }
}

template <class PopT>
struct SmallArgs {
  Scene<PopT, typename Prec<PopT>::Real> s;
  int cur, ns, listCap, redChunks, zlo, zend, seqFill;
  Plan *plan;
  lbm_sphere *sph;
  double *impAcc;
  long long slotCells, maxU;
  int2 *counts;
  int *fresh, *dead, *totals;
  double *partials, *dFluid, *dDead;
  unsigned *tickets;
  double rhoL, rhoG, gravity;
};

template <class PopT>
__global__ void kb_plan(const SmallArgs<PopT> *__restrict__ A) {
  const SmallArgs<PopT> &a = A[blockIdx.x];
  plan_body(a.plan, a.sph, a.ns, a.s.nx, a.s.ny, a.s.nz, a.impAcc, a.slotCells, a.maxU);
}
template <class PopT>
__global__ void kb_retag_box(const SmallArgs<PopT> *__restrict__ A) {
  const SmallArgs<PopT> &a = A[blockIdx.y];
  retag_box_body<PopT>(a.s, a.plan, blockIdx.x, gridDim.x);
}
template <class PopT>
__global__ void kb_compact_count(const SmallArgs<PopT> *__restrict__ A) {
  const SmallArgs<PopT> &a = A[blockIdx.y];
  compact_count_body(a.s.tag, a.s.tagPrev, a.s.nx, a.s.ny, a.plan, a.counts, blockIdx.x, gridDim.x);
}
template <class PopT>
__global__ void kb_compact_scan(const SmallArgs<PopT> *__restrict__ A) {
  const SmallArgs<PopT> &a = A[blockIdx.x];
  compact_scan_body(a.counts, a.plan, a.totals);
}
template <class PopT>
__global__ void kb_compact_emit(const SmallArgs<PopT> *__restrict__ A) {
  const SmallArgs<PopT> &a = A[blockIdx.y];
  compact_emit_body(a.s.tag, a.s.tagPrev, a.s.nx, a.s.ny, a.plan, a.counts, a.fresh, a.dead, a.listCap,
                    blockIdx.x, gridDim.x);
}
template <class PopT>
__global__ void __launch_bounds__(FILL_THREADS) kb_fresh_fill(const SmallArgs<PopT> *__restrict__ A) {
  const SmallArgs<PopT> &a = A[blockIdx.x];
  fresh_fill_body<PopT>(a.s, a.cur, a.fresh, a.totals, a.listCap, a.rhoL, a.rhoG, a.zlo, a.zend, a.seqFill);
}
template <class PopT>
__global__ void __launch_bounds__(RED_THREADS) kb_impulse_reduce(const SmallArgs<PopT> *__restrict__ A) {
  const SmallArgs<PopT> &a = A[blockIdx.z];
  if (a.ns == 0) return;
  impulse_reduce_body(&a.plan->ss, a.partials, a.redChunks, a.dFluid, a.tickets, blockIdx.x, blockIdx.y);
}
template <class PopT>
__global__ void __launch_bounds__(DEAD_THREADS) kb_absorb_dead(const SmallArgs<PopT> *__restrict__ A) {
  const SmallArgs<PopT> &a = A[blockIdx.y];
  if (a.ns == 0) return;
  absorb_dead_body(SceneFields<PopT>{a.s, a.cur}, a.s.nx, a.s.ny, a.dead, a.totals, a.listCap, a.rhoL, a.rhoG,
                   &a.plan->ss, a.dDead, blockIdx.x);
}
template <class PopT>
__global__ void kb_sphere_step(const SmallArgs<PopT> *__restrict__ A) {
  const SmallArgs<PopT> &a = A[blockIdx.x];
  if (a.ns == 0) return;
  sphere_step_body(a.sph, a.ns, a.gravity, a.dFluid, a.dDead, a.s.nx, a.s.ny, a.s.nz);
}

// ---------------------------------------------------------------- launcher

template <class PopT>
class Ops final : public OpsBase {
 public:
  using Real = typename Prec<PopT>::Real;
  using SceneT = Scene<PopT, Real>;

  size_t pop_bytes() const override { return sizeof(PopT); }
  size_t macro_bytes() const override { return sizeof(Real); }
  bool phases_supported() const override { return !Codec<PopT>::offset; }

  static SceneT scene(lbm_sim *h) {
    SceneT s;
    s.nx = h->nx;
    s.ny = h->ny;
    s.nz = h->nz;
    s.n = h->n;
    for (int c = 0; c < 2; c++) {
      s.F[c] = (PopT *)h->F[c];
      s.H[c] = (PopT *)h->H[c];
      s.phi[c] = (Real *)h->mac[c][0];
      s.rho[c] = (Real *)h->mac[c][1];
      s.ux[c] = (Real *)h->mac[c][2];
      s.uy[c] = (Real *)h->mac[c][3];
      s.uz[c] = (Real *)h->mac[c][4];
    }
    s.tag = h->tag;
    s.tagPrev = h->tagPrev;
    s.gx = (Real *)h->grad[0];
    s.gy = (Real *)h->grad[1];
    s.gz = (Real *)h->grad[2];
    s.lap = (Real *)h->grad[3];
    s.usx = (Real *)h->us[0];
    s.usy = (Real *)h->us[1];
    s.usz = (Real *)h->us[2];
    bool bfa = h->bfActive;
    s.bfx = bfa ? (Real *)h->bf[0] : nullptr;
    s.bfy = bfa ? (Real *)h->bf[1] : nullptr;
    s.bfz = bfa ? (Real *)h->bf[2] : nullptr;
    return s;
  }

  void init_flat(lbm_sim *h, const double *d_phiCol) override {
    k_init_flat<PopT><<<nblocks(h->n, 256), 256, 0, h->stream>>>(scene(h), d_phiCol);
    h->launches++;
  }
  void seed_hydrostatic(lbm_sim *h) override {
    long long cols = (long long)h->nx * h->nz;
    k_seed_hydrostatic<PopT><<<nblocks(cols, 128), 128, 0, h->stream>>>(
        scene(h), h->cur, h->params.rhoL, h->params.rhoG, h->params.gravity);
    h->launches++;
  }
  void gradients(lbm_sim *h) override {
    k_gradients<PopT><<<nblocks(h->n, 256), 256, 0, h->stream>>>(scene(h), h->cur);
    h->launches++;
  }
  void retag_full(lbm_sim *h) override {
    k_retag_full<PopT><<<nblocks(h->n, 256), 256, 0, h->stream>>>(scene(h), h->cur, &h->dPlan->ss);
    h->launches++;
  }
  void retag_mask(lbm_sim *h, const uint8_t *d_mask, const float *d_us) override {
    k_retag_mask<PopT><<<nblocks(h->n, 256), 256, 0, h->stream>>>(scene(h), h->cur, d_mask, d_us);
    h->launches++;
  }
  void link_count(lbm_sim *h, int *d_chunks) override {
    const unsigned chunks = nblocks(h->n, LINK_CHUNK);
    k_link_count<<<chunks, LINK_CHUNK, 0, h->stream>>>(h->tag, h->nx, h->ny, h->nz, h->n, d_chunks);
    k_link_scan<<<1, 1024, 0, h->stream>>>(d_chunks, (int)chunks);
    h->launches += 2;
  }
  void link_emit(lbm_sim *h, const int *d_chunks, int cap, int *cells, int8_t *dirs, double *mom) override {
    k_link_emit<PopT><<<nblocks(h->n, LINK_CHUNK), LINK_CHUNK, 0, h->stream>>>(scene(h), h->cur, d_chunks, cap,
                                                                                cells, dirs, mom);
    h->launches++;
  }
  void collide_phase(lbm_sim *h) override {
    k_collide_phase<PopT><<<nblocks(h->n, 256), 256, 0, h->stream>>>(scene(h), h->cur,
                                                                       make_const(h->params));
    h->launches++;
  }
  void stream_phase(lbm_sim *h) override {
    k_stream_phase<PopT><<<nblocks(h->n, 256), 256, 0, h->stream>>>(scene(h), h->cur);
    h->launches++;
  }
  void collide_hydro(lbm_sim *h) override {
    k_collide_hydro<PopT><<<nblocks(h->n, 256), 256, 0, h->stream>>>(scene(h), h->cur,
                                                                       make_const(h->params));
    h->launches++;
  }
  void stream_hydro_macro(lbm_sim *h) override {
    k_stream_hydro_macro<PopT><<<nblocks(h->n, 256), 256, 0, h->stream>>>(
        scene(h), h->cur, make_const(h->params), &h->dPlan->ss);
    h->launches++;
  }
  void retag_box(lbm_sim *h, long long maxCells) override {
    if (maxCells <= 0) return;
    k_retag_box<PopT><<<std::min(nblocks(maxCells, 256), SWEEP_CTAS), 256, 0, h->stream>>>(scene(h), h->dPlan);
    h->launches++;
  }
  void fresh_fill(lbm_sim *h) override {
    k_fresh_fill<PopT><<<1, FILL_THREADS, 0, h->stream>>>(scene(h), h->cur, h->fresh, h->totals,
                                                           (int)h->listCap, h->params.rhoL, h->params.rhoG,
                                                           h->slab ? h->ownLo : 0, h->slab ? h->ownHi + 1 : 0,
                                                           h->sequentialFill ? 1 : 0);
    h->launches++;
  }
  void absorb_dead(lbm_sim *h, double *d_out) override {
    const int ns = h->hPlan.ss.nsph > 0 ? h->hPlan.ss.nsph : 1;
    k_absorb_dead_scene<PopT><<<ns, DEAD_THREADS, 0, h->stream>>>(scene(h), h->cur, h->dead, h->totals,
                                                                  (int)h->listCap, h->params.rhoL,
                                                                  h->params.rhoG, &h->dPlan->ss, d_out);
    h->launches++;
  }

  // Tile shapes: rows 2, 4, 8 (the plain form, every storage form), and rows
  // 4 or 6 | LBM_FUSED_COMPACT / LBM_FUSED_ASYNC / LBM_FUSED_STAGED (the
  // compact-ring forms, which keep FP32 values in their ring: FP32, FP16 and
  // BF16 storage); SHAPE_WIDE marks a launch over a grid whose populations
  // need 64-bit offsets.  f(IC<rows>, IC<form>, wide) is called with the
  // shape's compile-time launch form: 0 plain, PIPE_STAGED, PIPE_COMPACT,
  // PIPE_ASYNC.
  template <class F>
  static void with_shape(int shape, F &&f) {
    const bool wide = (shape & SHAPE_WIDE) != 0;
    auto go = [&](auto T, auto S) {
      if (wide) f(T, S, std::true_type{});
      else f(T, S, std::false_type{});
    };
    auto pipe = [&](auto T, auto S) {
      if constexpr (kPipe) go(T, S);
      else go(IC<4>{}, IC<0>{});  // not reached: shape_ok refuses these shapes
    };
    switch (shape & ~SHAPE_WIDE) {
      case 2: go(IC<2>{}, IC<0>{}); break;
      case 4: go(IC<4>{}, IC<0>{}); break;
      case 4 | LBM_FUSED_COMPACT: pipe(IC<4>{}, IC<PIPE_COMPACT>{}); break;
      case 6 | LBM_FUSED_COMPACT: pipe(IC<6>{}, IC<PIPE_COMPACT>{}); break;
      case 4 | LBM_FUSED_ASYNC: pipe(IC<4>{}, IC<PIPE_ASYNC>{}); break;
      case 6 | LBM_FUSED_ASYNC: pipe(IC<6>{}, IC<PIPE_ASYNC>{}); break;
      case 4 | LBM_FUSED_STAGED: pipe(IC<4>{}, IC<PIPE_STAGED>{}); break;
      case 6 | LBM_FUSED_STAGED: pipe(IC<6>{}, IC<PIPE_STAGED>{}); break;
      case TMA_ROWS | LBM_FUSED_TMA: pipe(IC<TMA_ROWS>{}, IC<PIPE_TMA>{}); break;
      case TMA_ROWS | LBM_FUSED_L2PF: pipe(IC<TMA_ROWS>{}, IC<PIPE_L2PF>{}); break;
      default: go(IC<8>{}, IC<0>{}); break;
    }
  }
  static constexpr bool kPipe = sizeof(Real) == 4;
  bool shape_ok(int shape) const override {
    if (shape == 2 || shape == 4 || shape == 8) return true;
    const int rows = shape & 0xff, form = shape & ~0xff;
    if (form == LBM_FUSED_TMA || form == LBM_FUSED_L2PF) return kPipe && rows == TMA_ROWS;
    return kPipe && (rows == 4 || rows == 6) &&
           (form == LBM_FUSED_COMPACT || form == LBM_FUSED_ASYNC || form == LBM_FUSED_STAGED);
  }
  // shared memory, warps and kernels of a launch form
  template <int TY, int FORM>
  static constexpr size_t smem_of() {
    if constexpr (FORM == 0) return FusedSmem<PopT, TY>::bytes;
    else return PipeSmem<PopT, TY, FORM>::bytes;
  }
  template <int TY, int FORM>
  static constexpr int warps_of() {
    if constexpr (FORM == 0) return FusedSmem<PopT, TY>::warps;
    else return PipeSmem<PopT, TY, FORM>::warps;
  }
  template <int TY, int FORM, bool WIDE, bool PACK = false>
  static auto step_kernel() {
    if constexpr (FORM == 0) return k_fused_step<PopT, TY, WIDE, PACK>;
    else return k_fused_pipe<PopT, TY, FORM, WIDE, PACK>;
  }
  template <int TY, int FORM, bool WIDE>
  static auto batch_kernel() {
    if constexpr (FORM == 0) return k_fused_batch<PopT, TY, WIDE>;
    else return k_fused_pipe_batch<PopT, TY, FORM, WIDE>;
  }

  template <int TY, int STG, bool WIDE>
  void launch_fused(lbm_sim *h, const FusedArgs<PopT> &a, int zchunk) {
    if (a.pack) launch_fused_as<TY, STG, WIDE, true>(h, a, zchunk);
    else launch_fused_as<TY, STG, WIDE, false>(h, a, zchunk);
  }
  template <int TY, int STG, bool WIDE, bool PACK>
  void launch_fused_as(lbm_sim *h, const FusedArgs<PopT> &a, int zchunk) {
    constexpr size_t smem = smem_of<TY, STG>();
    const auto kern = step_kernel<TY, STG, WIDE, PACK>();
    // the shared-memory opt-in is per device
    static unsigned long long attrSet = 0;
    const unsigned long long bit = 1ull << (h->device & 63);
    if (!(attrSet & bit)) {
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      attrSet |= bit;
    }
    dim3 block(32, warps_of<TY, STG>());  // TY cell warps and the halo warps
    dim3 grid((h->nx + 31) / 32, (h->ny + TY - 1) / TY, (h->nz - 2 + zchunk - 1) / zchunk);
    kern<<<grid, block, smem, h->stream>>>(a);
    h->launches++;
  }

  FusedArgs<PopT> make_args(lbm_sim *h, int cur, int zchunk) {
    FusedArgs<PopT> a;
    a.s = scene(h);
    a.cur = cur;
    a.zchunk = zchunk;
    StepConst k = make_const(h->params);
    a.om = k.invTau;
    a.omP = k.invTauPhi;
    a.A = k.A;
    a.beta4 = 4 * k.beta;
    a.kappa = k.kappa;
    a.rhoG = k.rhoG;
    a.dRho = k.dRho;
    a.gravity = k.gravity;
    a.sharpC4 = 4 * k.sharpC;
    a.ss = &h->dPlan->ss;
    a.status = h->totals + 2;
    a.withhold = h->withholdStage ? 1 : 0;
    a.pack = h->fusePack;
    a.maps = (const StageMaps *)h->dMaps;
    return a;
  }
  size_t fused_args_bytes() const override { return sizeof(FusedArgs<PopT>); }
  void fused_args(lbm_sim *h, int cur, int zchunk, void *out) override {
    FusedArgs<PopT> a = make_args(h, cur, zchunk);
    memcpy(out, &a, sizeof(a));
  }
  template <int TY, int STG, bool WIDE>
  int batch_ctas(int device) {
    constexpr size_t smem = smem_of<TY, STG>();
    const auto kern = batch_kernel<TY, STG, WIDE>();
    static unsigned long long attrSet = 0;
    const unsigned long long bit = 1ull << (device & 63);
    if (!(attrSet & bit)) {
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      attrSet |= bit;
    }
    int per = 0, sms = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, 32 * warps_of<TY, STG>(), smem);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    return std::max(1, per) * std::max(1, sms);
  }
  int build_stage_maps(lbm_sim *h) override {
    if (!kPipe || h->nx % 16 != 0) return LBM_OK;
    const auto enc = tensor_map_encoder();
    if (!enc) return LBM_OK;
    StageMaps m;
    memset(&m, 0, sizeof(m));
    const cuuint64_t nx = h->nx, ny = h->ny, nz = h->nz, pb = sizeof(PopT), rb = sizeof(float);
    const CUtensorMapDataType popType =
        sizeof(PopT) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_UINT16;
    bool ok = true;
    auto map = [&](TensorMap *out, CUtensorMapDataType type, int rank, void *base, const cuuint64_t *dims,
                   const cuuint64_t *strides, const cuuint32_t *box) {
      const cuuint32_t unit[5] = {1, 1, 1, 1, 1};
      ok = ok && enc(reinterpret_cast<CUtensorMap *>(out), type, (cuuint32_t)rank, base, dims, strides, box,
                     unit, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    };
    constexpr cuuint32_t TY = TMA_ROWS;
    // populations: (elements of a block, blocks of a row, y, z); box 4 blocks x TY rows
    const cuuint64_t b27 = PopGroups<Q27>::BLOCK, b7 = PopGroups<Q7>::BLOCK;
    const cuuint64_t dF[4] = {b27, nx / 8, ny, nz}, sF[3] = {b27 * pb, nx / 8 * b27 * pb, ny * nx / 8 * b27 * pb};
    const cuuint64_t dH[4] = {b7, nx / 8, ny, nz}, sH[3] = {b7 * pb, nx / 8 * b7 * pb, ny * nx / 8 * b7 * pb};
    const cuuint32_t bF[4] = {(cuuint32_t)b27, 4, TY, 1}, bH[4] = {(cuuint32_t)b7, 4, TY, 1};
    // cell arrays: (x, y, z); box 32 x TY, phi 40 x (TY + 2)
    const cuuint64_t d3[3] = {nx, ny, nz}, sR[2] = {nx * rb, nx * ny * rb}, sT[2] = {nx, nx * ny};
    const cuuint32_t bRow[3] = {32, TY, 1}, bPhi[3] = {40, TY + 2, 1};
    for (int c = 0; c < 2; c++) {
      map(&m.f[c], popType, 4, h->F[c], dF, sF, bF);
      map(&m.h[c], popType, 4, h->H[c], dH, sH, bH);
      map(&m.phi[c], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, h->mac[c][0], d3, sR, bPhi);
      map(&m.rho[c], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, h->mac[c][1], d3, sR, bRow);
      map(&m.ux[c], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, h->mac[c][2], d3, sR, bRow);
      map(&m.uy[c], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, h->mac[c][3], d3, sR, bRow);
      map(&m.uz[c], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, h->mac[c][4], d3, sR, bRow);
    }
    map(&m.tag, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, h->tag, d3, sT, bRow);
    if (!ok) return LBM_OK;  // no maps: the form runs as the compact one
    void *d = nullptr;
    if (cudaMallocAsync(&d, sizeof(StageMaps), h->stream) != cudaSuccess) {
      cudaGetLastError();
      return LBM_ERR_OOM;
    }
    if (cudaMemcpyAsync(d, &m, sizeof(StageMaps), cudaMemcpyHostToDevice, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess) {
      cudaFreeAsync(d, h->stream);
      return LBM_ERR_CUDA;
    }
    h->dMaps = d;
    return LBM_OK;
  }
  bool u_in_pads() const override { return Scene<PopT, Real>::UPAD; }
  void u_array(lbm_sim *h, int comp, int half, void *arr, bool toScene) override {
    k_u_array<PopT><<<nblocks(h->n, 256), 256, 0, h->stream>>>(scene(h), comp, half, (Real *)arr, toScene ? 1 : 0);
    h->launches++;
  }
  size_t small_args_bytes() const override { return sizeof(SmallArgs<PopT>); }
  void small_args(lbm_sim *h, int cur, int ns, long long slotCells, long long maxU, int redChunks,
                  void *out) override {
    SmallArgs<PopT> a;
    memset(&a, 0, sizeof(a));
    a.s = scene(h);
    a.cur = cur;
    a.ns = ns;
    a.listCap = (int)h->listCap;
    a.redChunks = redChunks;
    a.zlo = h->slab ? h->ownLo : 0;
    a.zend = h->slab ? h->ownHi + 1 : 0;
    a.seqFill = h->sequentialFill ? 1 : 0;
    a.plan = h->dPlan;
    a.sph = h->dSph;
    a.impAcc = h->impAcc;
    a.slotCells = slotCells;
    a.maxU = maxU;
    a.counts = h->counts;
    a.fresh = h->fresh;
    a.dead = h->dead;
    a.totals = h->totals;
    a.partials = h->partials;
    a.dFluid = h->dOut;
    a.dDead = h->dOut + LBM_MAX_SPHERES * 6;
    a.tickets = h->redTickets;
    a.rhoL = h->params.rhoL;
    a.rhoG = h->params.rhoG;
    a.gravity = h->params.gravity;
    memcpy(out, &a, sizeof(a));
  }
  void batch_pre(const void *d_small, int n, unsigned retagCtas, unsigned compactCtas, cudaStream_t st) override {
    const auto *A = (const SmallArgs<PopT> *)d_small;
    kb_plan<PopT><<<n, 32, 0, st>>>(A);
    kb_retag_box<PopT><<<dim3(retagCtas, n), 256, 0, st>>>(A);
    kb_compact_count<PopT><<<dim3(compactCtas, n), COMPACT_THREADS, 0, st>>>(A);
    kb_compact_scan<PopT><<<n, 1024, 0, st>>>(A);
    kb_compact_emit<PopT><<<dim3(compactCtas, n), COMPACT_THREADS, 0, st>>>(A);
    kb_fresh_fill<PopT><<<n, FILL_THREADS, 0, st>>>(A);
  }
  void batch_post(const void *d_small, int n, int redChunks, int maxSpheres, cudaStream_t st) override {
    if (maxSpheres <= 0) return;
    const auto *A = (const SmallArgs<PopT> *)d_small;
    kb_impulse_reduce<PopT><<<dim3(redChunks, maxSpheres, n), RED_THREADS, 0, st>>>(A);
    kb_absorb_dead<PopT><<<dim3(maxSpheres, n), DEAD_THREADS, 0, st>>>(A);
    kb_sphere_step<PopT><<<n, 32, 0, st>>>(A);
  }
  void warm(int device) override {
    static const int shapes[] = {2, 4, 8, 4 | LBM_FUSED_COMPACT, 6 | LBM_FUSED_COMPACT, 4 | LBM_FUSED_ASYNC,
                                 6 | LBM_FUSED_ASYNC, 4 | LBM_FUSED_STAGED, 6 | LBM_FUSED_STAGED,
                                 TMA_ROWS | LBM_FUSED_TMA, TMA_ROWS | LBM_FUSED_L2PF};
    for (int sh : shapes) {
      if (!shape_ok(sh)) continue;
      with_shape(sh, [&](auto T, auto S, auto W) {
        constexpr int TY = decltype(T)::value, FORM = decltype(S)::value;
        constexpr bool WIDE = decltype(W)::value;
        batch_ctas<TY, FORM, WIDE>(device);
        cudaFuncSetAttribute(step_kernel<TY, FORM, WIDE>(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem_of<TY, FORM>());
        cudaFuncSetAttribute(step_kernel<TY, FORM, WIDE, true>(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem_of<TY, FORM>());
      });
    }
    cudaGetLastError();
  }
  int fused_batch_ctas(int shape, int device) override {
    int r = 0;
    with_shape(shape, [&](auto T, auto S, auto W) {
      r = batch_ctas<decltype(T)::value, decltype(S)::value, decltype(W)::value>(device);
    });
    return r;
  }
  void fused_batch(const void *d_args, const int *d_tileStart, const int3 *d_tileGrid, int nscenes, int shape,
                   int ctas, cudaStream_t st) override {
    with_shape(shape, [&](auto T, auto S, auto W) {
      constexpr int TY = decltype(T)::value;
      constexpr int FORM = decltype(S)::value;
      dim3 block(32, warps_of<TY, FORM>());
      batch_kernel<TY, FORM, decltype(W)::value>()<<<ctas, block, smem_of<TY, FORM>(), st>>>(
          (const FusedArgs<PopT> *)d_args, d_tileStart, d_tileGrid, nscenes);
    });
  }

  void fused_step(lbm_sim *h, const FusedCfg &cfg) override {
    FusedArgs<PopT> a = make_args(h, h->cur, cfg.zchunk);
    const int shape = resolve_shape(h, cfg.ty) | (needs_wide(h->n) ? SHAPE_WIDE : 0);
    with_shape(shape, [&](auto T, auto S, auto W) {
      launch_fused<decltype(T)::value, decltype(S)::value, decltype(W)::value>(h, a, cfg.zchunk);
    });
  }

  cudaError_t read_fault(lbm_sim *h, unsigned long long out[4]) override {
    cudaError_t e = cudaMemcpyFromSymbolAsync(out, lbm_fault_word, 4 * sizeof(unsigned long long), 0,
                                              cudaMemcpyDeviceToHost, h->stream);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return e;
    static const unsigned long long zero[4] = {0, 0, 0, 0};
    return cudaMemcpyToSymbol(lbm_fault_word, zero, sizeof(zero));
  }

  size_t fused_smem(int shape) const override {
    size_t r = 0;
    with_shape(shape, [&](auto T, auto S, auto) { r = smem_of<decltype(T)::value, decltype(S)::value>(); });
    return r;
  }

  void pack(lbm_sim *h, uint8_t *d_out) override {
    k_pack<PopT><<<nblocks(h->n, 256), 256, 0, h->stream>>>(scene(h), h->cur, d_out);
    h->launches++;
  }
  void pack_end_planes(lbm_sim *h, uint8_t *d_out) override {
    const long long cells = 2LL * h->nx * h->ny;
    k_pack_end_planes<PopT><<<nblocks(cells, 256), 256, 0, h->stream>>>(scene(h), h->cur, d_out);
    h->launches++;
  }
  void watch_finite(lbm_sim *h, unsigned long long *d_first) override {
    k_watch_finite<PopT><<<std::min(nblocks(h->n, 256), 148u * 8u), 256, 0, h->stream>>>(scene(h), h->cur,
                                                                                        d_first);
    h->launches++;
  }
  void upload_pops(lbm_sim *h, bool isH, int half, const float *d_aos, long long c0,
                   long long cells) override {
    k_aos_to_soa<PopT><<<nblocks(cells, 256), 256, 0, h->stream>>>(scene(h), isH ? 1 : 0, half,
                                                                     h->cur, d_aos, c0, cells);
    h->launches++;
  }
  void download_pops(lbm_sim *h, bool isH, int half, float *d_aos, long long c0,
                     long long cells) override {
    int src = half == 2 ? 1 - h->cur : h->cur;
    k_soa_to_aos<PopT, float><<<nblocks(cells, 256), 256, 0, h->stream>>>(scene(h), isH ? 1 : 0, src,
                                                                            d_aos, c0, cells);
    h->launches++;
  }
  void download_pops64(lbm_sim *h, bool isH, int half, double *d_aos, long long c0,
                       long long cells) override {
    int src = half == 2 ? 1 - h->cur : h->cur;
    k_soa_to_aos<PopT, double><<<nblocks(cells, 256), 256, 0, h->stream>>>(scene(h), isH ? 1 : 0, src,
                                                                             d_aos, c0, cells);
    h->launches++;
  }
  void reencode_h(lbm_sim *h, int half, const void *d_oldPhi) override {
    if (!Codec<PopT>::offset) return;
    k_reencode_h<PopT><<<nblocks(h->n, 256), 256, 0, h->stream>>>(scene(h), half,
                                                                    (const Real *)d_oldPhi);
    h->launches++;
  }
  void sphere_step_device(lbm_sim *h, lbm_sphere *d_sph, int nsph, double gravity,
                          const double *d_fluid, const double *d_dead) override {
    k_sphere_step<<<1, 32, 0, h->stream>>>(d_sph, nsph, gravity, d_fluid, d_dead, h->nx, h->ny, h->nz);
    h->launches++;
  }
};

}  // namespace lbm
