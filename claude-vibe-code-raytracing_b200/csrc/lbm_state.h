// Host-side state of one scene handle and the per-storage-type kernel
// launcher interface.  Shared by the C ABI (lbm_capi.cu) and the typed
// launchers (lbm_inst_*.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "lbm_b200.h"
#include "lbm_core.cuh"

struct lbm_sim;

namespace lbm {

// Launch configuration of the fused step kernel.
struct FusedCfg {
  int ty = 4;       // tile shape: cell rows per CTA (CTA = 32 x (rows + 2) threads),
                    // | LBM_FUSED_COMPACT / _ASYNC / _STAGED / _TMA for the compact-ring forms
  int zchunk = 32;  // z planes marched per CTA
};

// cell rows per CTA of a tile shape
inline int shape_rows(int shape) { return shape & 0xff; }
// internal shape bit: the launch covers a grid whose D3Q27 populations exceed
// 2^31 elements, so the fused kernel uses 64-bit population offsets
constexpr int SHAPE_WIDE = 0x200;
inline bool needs_wide(long long cells) { return pop_elems(cells, 27) >= (1LL << 31) - 64; }


class OpsBase {
 public:
  virtual ~OpsBase() {}
  virtual size_t pop_bytes() const = 0;    // bytes per stored population
  virtual size_t macro_bytes() const = 0;  // bytes per macro value
  virtual bool phases_supported() const = 0;
  virtual void init_flat(lbm_sim *h, const double *d_phiCol) = 0;
  virtual void seed_hydrostatic(lbm_sim *h) = 0;
  virtual void gradients(lbm_sim *h) = 0;
  // Kernels of a step read the sphere set and boxes from h->dPlan.
  virtual void retag_full(lbm_sim *h) = 0;
  // retag from a host-evaluated solid mask and surface velocities (device copies)
  virtual void retag_mask(lbm_sim *h, const uint8_t *d_mask, const float *d_us) = 0;
  // momentum-exchange links of the last phase-by-phase hydro stream, scan order
  virtual void link_count(lbm_sim *h, int *d_chunks) = 0;
  virtual void link_emit(lbm_sim *h, const int *d_chunks, int cap, int *cells, int8_t *dirs, double *mom) = 0;
  virtual void collide_phase(lbm_sim *h) = 0;
  virtual void stream_phase(lbm_sim *h) = 0;
  virtual void collide_hydro(lbm_sim *h) = 0;
  virtual void stream_hydro_macro(lbm_sim *h) = 0;
  virtual void retag_box(lbm_sim *h, long long maxCells) = 0;
  virtual void fresh_fill(lbm_sim *h) = 0;
  virtual void absorb_dead(lbm_sim *h, double *d_out) = 0;
  virtual void fused_step(lbm_sim *h, const FusedCfg &cfg) = 0;
  virtual void pack(lbm_sim *h, uint8_t *d_out) = 0;
  virtual void pack_end_planes(lbm_sim *h, uint8_t *d_out) = 0;
  virtual void watch_finite(lbm_sim *h, unsigned long long *d_first) = 0;
  // Reference-layout float32 <-> device storage for population fields.
  // half: 0 = both halves (current state), 1 = [cur], 2 = [1-cur].
  virtual void upload_pops(lbm_sim *h, bool isH, int half, const float *d_aos, long long c0,
                           long long cells) = 0;
  virtual void download_pops(lbm_sim *h, bool isH, int half, float *d_aos, long long c0,
                             long long cells) = 0;
  virtual void download_pops64(lbm_sim *h, bool isH, int half, double *d_aos, long long c0,
                               long long cells) = 0;
  // Re-express h offsets after phi changed from d_oldPhi (both halves).
  virtual void reencode_h(lbm_sim *h, int half, const void *d_oldPhi) = 0;
  virtual void sphere_step_device(lbm_sim *h, lbm_sphere *d_sph, int nsph, double gravity,
                                  const double *d_fluid, const double *d_dead) = 0;
  // Fused-step kernel geometry (for the bench and the autotuner).
  virtual size_t fused_smem(int ty) const = 0;
  // Batched fused step: per-scene descriptors (FusedArgs of this storage type,
  // fused_args_bytes() each) for a given ping-pong half, and one persistent
  // launch over the tiles of every scene.
  virtual size_t fused_args_bytes() const = 0;
  virtual void fused_args(lbm_sim *h, int cur, int zchunk, void *out) = 0;
  virtual int fused_batch_ctas(int ty, int device) = 0;  // resident CTAs on the device
  virtual void fused_batch(const void *d_args, const int *d_tileStart, const int3 *d_tileGrid,
                           int nscenes, int ty, int ctas, cudaStream_t st) = 0;
  // Fault record of the bounds-checked build (all zero otherwise); cleared on read.
  virtual cudaError_t read_fault(lbm_sim *h, unsigned long long out[4]) = 0;
  // a tile shape this storage form supports (rows 2, 4, 8; 4 | LBM_FUSED_STAGED for FP16/BF16)
  virtual bool shape_ok(int shape) const = 0;
  // load every fused step and batch kernel instance of this storage form on
  // the device (and set their shared-memory opt-in), so that no first launch
  // waits for a module load
  virtual void warm(int device) = 0;
  // ux and uy held in the population pad slots (FP32 / FP64 storage), and
  // their copy to or from a plain array of one half (the field transfers)
  virtual bool u_in_pads() const = 0;
  virtual void u_array(lbm_sim *h, int comp, int half, void *arr, bool toScene) = 0;
  // a batch's sparse kernels, one launch per kind for all scenes: the
  // per-scene argument block, then the kernels before and after the fused
  // launch over a device table of n such blocks
  virtual size_t small_args_bytes() const = 0;
  virtual void small_args(lbm_sim *h, int cur, int ns, long long slotCells, long long maxU, int redChunks,
                          void *out) = 0;
  virtual void batch_pre(const void *d_small, int n, unsigned retagCtas, unsigned compactCtas,
                         cudaStream_t st) = 0;
  virtual void batch_post(const void *d_small, int n, int redChunks, int maxSpheres, cudaStream_t st) = 0;
  // the tensor maps of the TMA-staged form (h->dMaps), where the storage
  // form and the grid allow them (nx a multiple of 16); none otherwise
  virtual int build_stage_maps(lbm_sim *) { return 0; }
};

OpsBase *make_ops_f32();
OpsBase *make_ops_f16();
OpsBase *make_ops_bf16();
OpsBase *make_ops_f64();

}  // namespace lbm

struct lbm_sim {
  int nx = 0, ny = 0, nz = 0, storage = 0, device = 0;
  long long n = 0;
  cudaStream_t stream = nullptr;
  lbm_params params{};
  int cur = 0;
  lbm::OpsBase *ops = nullptr;
  lbm::FusedCfg cfg;
  bool fusedOK = true;  // the fused kernel's 32-bit indexing covers this grid
  bool withholdStage = false;  // test hook: the staged fused kernel withholds its first copy

  // device memory
  void *F[2] = {nullptr, nullptr};
  void *H[2] = {nullptr, nullptr};
  void *mac[2][5] = {{nullptr}};  // phi, rho, ux, uy, uz
  uint8_t *tag = nullptr, *tagPrev = nullptr;
  void *grad[4] = {nullptr};  // gx gy gz lap (phase-by-phase scratch)
  void *us[3] = {nullptr};
  void *bf[3] = {nullptr};
  bool bfActive = false;

  int *fresh = nullptr, *dead = nullptr;  // scan-ordered lists
  long long listCap = 0;
  int2 *counts = nullptr;
  long long countsCap = 0;
  int *totals = nullptr;  // device [3]: n_fresh, n_dead, fused-step status (non-zero: a bounded wait ran out)
  bool listsValid = false;

  double *impAcc = nullptr;  // per-cell impulse slots of every sphere
  long long impCap = 0;      // doubles
  double *partials = nullptr;
  void *dMaps = nullptr;    // tensor maps of the TMA-staged form (device memory), or null
  void *meshTri = nullptr;  // a mesh's triangles for lbm_voxelize_mesh / lbm_retag_cells_mesh
  size_t meshCap = 0;
  unsigned *redTickets = nullptr;  // [LBM_MAX_SPHERES] last-block tickets of the impulse reduction
  long long partialsCap = 0;  // doubles
  int partialsChunks = 0;
  double *dOut = nullptr;      // device [2][MAX][6]: fluid impulses, dead impulses
  double *hOut = nullptr;      // pinned host mirror
  lbm_sphere *dSph = nullptr;  // device sphere array for the coupled loop
  lbm::Plan hPlan{};           // host copy of the step plan
  lbm::Plan *dPlan = nullptr;  // device step plan read by the kernels
  void *staging = nullptr;
  size_t stagingBytes = 0;
  void *image = nullptr;  // rendered RGBA8 frame (lbm_render)
  // lbm_pack_volume_async / lbm_step_frame: packed frames on the device, two
  // used in turn, each copied to the host on copyStream; evPacked orders a
  // copy after its pack, evFrame[b] the next pack into buffer b after b's
  // copy, evCopied marks the last copy issued
  void *frameDev[2] = {nullptr, nullptr};
  cudaEvent_t evFrame[2] = {nullptr, nullptr};
  cudaEvent_t evPackedSlot[2] = {nullptr, nullptr};
  bool framePending[2] = {false, false};
  int frameNext = 0;
  // lbm_step_frame's copy to the host, issued when the next step's fused
  // kernel is queued (so it runs beside that kernel, not ahead of the step's
  // small read-backs on the same copy engine); -1: none waiting
  int deferredSlot = -1;
  uint8_t *deferredHost = nullptr;
  cudaStream_t copyStream = nullptr;
  cudaEvent_t evPacked = nullptr, evCopied = nullptr;
  bool copyPending = false;
  size_t imageBytes = 0;
  double *dPhiCol = nullptr;
  int *hTotals = nullptr;  // pinned [3]
  // NaN/Inf watchdog (lbm_set_nan_watchdog): off while watchEvery is 0
  int watchEvery = 0;
  long long watchSteps = 0;            // steps completed since the last scan
  unsigned long long *dWatch = nullptr;  // device: lowest non-finite cell index

  lbm::Box boxLast{{1, 1, 1}, {0, 0, 0}};
  lbm::Box boxLastLast{{1, 1, 1}, {0, 0, 0}};
  lbm::Box lastRetagBox{{1, 1, 1}, {0, 0, 0}};
  // a step split by lbm_step_begin / lbm_step_end: the spheres' box of the
  // begun step, and how many spheres it was begun with (-1: none begun)
  lbm::Box stepNow{{1, 1, 1}, {0, 0, 0}};
  // a frame step: the fused kernel writes the step's RG8 volume here
  // (planes 1 .. nz-2; pack_end_planes adds the two end planes), else null
  uint8_t *fusePack = nullptr;
  // test hook: fill fresh cells with one thread in list order
  bool sequentialFill = false;
  int stepBegunNs = -1;
  int fullRetagSteps = 0;
  int nsphLast = 0;

  // z slab of a larger scene (lbm_set_slab): local plane k is global plane
  // k + zoff; planes [ownLo, ownHi] are this handle's, the others copies of
  // its neighbours' (slab = false: the whole grid is the scene)
  bool slab = false;
  int zoff = 0, ownLo = 0, ownHi = 0;

  int *linkChunks = nullptr;  // generic-solid link compaction: per-chunk counts, then offsets
  long long linkChunksCap = 0;
  void *linkBuf = nullptr;  // the link list (cells, moms, dirs) on the device
  long long linkBufCap = 0;  // links

  size_t deviceBytes = 0;
  long long launches = 0;
  unsigned long long h2dBytes = 0, d2hBytes = 0;
  std::string err;

  // absorbDeadCells computed by the step that precedes it (lbm_step_end)
  // and fetched with the step's impulses: the result, the spheres it was
  // computed for, and the handle's launch and transfer counts, parameters and
  // current half when it was taken.  lbm_absorb_dead_cells returns it while
  // all of these still match; anything that moves device state in between
  // either changes them or clears `valid` itself.
  struct DeadAhead {
    bool valid = false;
    int ns = 0;
    lbm_sphere sp[LBM_MAX_SPHERES];
    double out[LBM_MAX_SPHERES * 6];
    long long launches = 0;
    unsigned long long h2d = 0, d2h = 0;
    lbm_params params;
    int cur = 0;
  } deadAhead;

  // CUDA-event timing of the fused kernel (lbm_fused_timing)
  bool timing = false;
  std::vector<cudaEvent_t> evStart, evStop;
  size_t evUsed = 0;
};

namespace lbm {
// the tile shape a fused launch of `shape` on this handle uses: the
// TMA-staged and L2-prefetch forms need the scene's tensor maps (nx a
// multiple of 16), otherwise the compact form of the same rows
inline int resolve_shape(const lbm_sim *h, int shape) {
  if ((shape & (LBM_FUSED_TMA | LBM_FUSED_L2PF)) && !h->dMaps)
    return shape_rows(shape) | LBM_FUSED_COMPACT | (shape & SHAPE_WIDE);
  return shape;
}
}  // namespace lbm
