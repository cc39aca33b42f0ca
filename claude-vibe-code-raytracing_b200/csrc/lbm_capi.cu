// C ABI of the B200-native LBM step (declarations and reference citations in
// include/lbm_b200.h).  Host orchestration only: allocation, field transfers,
// the sphere bounding boxes, and the launch sequence of every entry point.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "lbm_kernels.cuh"
#include "lbm_mesh.cuh"
#include "lbm_render.h"
#include "lbm_sphere.cuh"
#include "lbm_state.h"

using namespace lbm;

namespace {

int fail(lbm_sim *h, int code, const std::string &msg) {
  if (h) h->err = msg;
  return code;
}

int cuda_fail(lbm_sim *h, const char *what, cudaError_t e) {
  cudaGetLastError();  // clear a sticky-free error so the handle stays usable
  return fail(h, e == cudaErrorMemoryAllocation ? LBM_ERR_OOM : LBM_ERR_CUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                            \
  do {                                                      \
    cudaError_t e_ = (call);                                \
    if (e_ != cudaSuccess) return cuda_fail(h, #call, e_); \
  } while (0)

#define CKL(what)                                           \
  do {                                                      \
    cudaError_t e_ = cudaGetLastError();                    \
    if (e_ != cudaSuccess) return cuda_fail(h, what, e_);   \
  } while (0)

OpsBase *ops_for(int storage) {
  switch (storage) {
    case LBM_STORE_F32: return make_ops_f32();
    case LBM_STORE_F16: return make_ops_f16();
    case LBM_STORE_BF16: return make_ops_bf16();
    case LBM_STORE_F64: return make_ops_f64();
  }
  return nullptr;
}

size_t pop_bytes_of(int storage) {
  return storage == LBM_STORE_F64 ? 8 : storage == LBM_STORE_F32 ? 4 : 2;
}
size_t mac_bytes_of(int storage) { return storage == LBM_STORE_F64 ? 8 : 4; }


// Device memory comes from the device's stream-ordered pool, allocated and
// freed on the handle's stream: creating or destroying a scene does not stop
// the device (a plain cudaFree waits for every stream), so a server can admit
// and retire scenes while others step.  The pool keeps freed memory for the
// next scene (release threshold raised once per device).
void keep_pool(int device) {
  static std::mutex mu;
  static unsigned long long done = 0;
  std::lock_guard<std::mutex> lk(mu);
  const unsigned long long bit = 1ull << (device & 63);
  if (done & bit) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  cudaGetLastError();
  done |= bit;
}

int dalloc(lbm_sim *h, void **p, size_t bytes) {
  cudaError_t e = cudaMallocAsync(p, bytes, h->stream);
  if (e != cudaSuccess) {
    *p = nullptr;
    return cuda_fail(h, "cudaMallocAsync", e);
  }
  h->deviceBytes += bytes;
  return LBM_OK;
}

#define DALLOC(ptr, bytes)                                        \
  do {                                                            \
    int rc_ = dalloc(h, (void **)&(ptr), (size_t)(bytes));        \
    if (rc_ != LBM_OK) return rc_;                                \
  } while (0)

// Every host<->device copy of the ABI goes through here and is counted
// (lbm_transfer_bytes), so callers can report the bytes a step moves.
cudaError_t copy_async(lbm_sim *h, void *dst, const void *src, size_t bytes, cudaMemcpyKind kind,
                       cudaStream_t s) {
  if (kind == cudaMemcpyHostToDevice) h->h2dBytes += bytes;
  if (kind == cudaMemcpyDeviceToHost) h->d2hBytes += bytes;
  return cudaMemcpyAsync(dst, src, bytes, kind, s);
}

int ensure_staging(lbm_sim *h, size_t bytes) {
  if (h->stagingBytes >= bytes) return LBM_OK;
  if (h->staging) {
    cudaFreeAsync(h->staging, h->stream);
    h->deviceBytes -= h->stagingBytes;
    h->staging = nullptr;
    h->stagingBytes = 0;
  }
  DALLOC(h->staging, bytes);
  h->stagingBytes = bytes;
  return LBM_OK;
}

int ensure_scalar(lbm_sim *h, void **arr) {
  if (*arr) return LBM_OK;
  size_t bytes = (size_t)h->n * h->ops->macro_bytes();
  DALLOC(*arr, bytes);
  CK(cudaMemsetAsync(*arr, 0, bytes, h->stream));
  return LBM_OK;
}

int ensure_phase_scratch(lbm_sim *h) {
  for (int a = 0; a < 4; a++) {
    int rc = ensure_scalar(h, &h->grad[a]);
    if (rc) return rc;
  }
  for (int a = 0; a < 3; a++) {
    int rc = ensure_scalar(h, &h->us[a]);
    if (rc) return rc;
  }
  return LBM_OK;
}

Box interior(const lbm_sim *h) {
  Box b;
  b.lo[0] = b.lo[1] = b.lo[2] = 1;
  b.hi[0] = h->nx - 2;
  b.hi[1] = h->ny - 2;
  b.hi[2] = h->nz - 2;
  return b;
}

Box spheres_box(const lbm_sim *h, const lbm_sphere *sp, int ns) {
  Box u{{1, 1, 1}, {0, 0, 0}};
  for (int b = 0; b < ns; b++)
    u = box_union(u, sphere_box(sp[b].cx, sp[b].cy, sp[b].cz - h->zoff, sp[b].r, h->nx, h->ny, h->nz));
  return u;
}

int check_spheres(lbm_sim *h, const lbm_sphere *sp, int ns) {
  if (ns < 0 || ns > LBM_MAX_SPHERES) return fail(h, LBM_ERR_ARG, "nspheres out of range");
  if (ns > 0 && !sp) return fail(h, LBM_ERR_ARG, "spheres is NULL");
  return LBM_OK;
}

int upload_plan(lbm_sim *h) {
  // pageable source: the copy is staged before cudaMemcpyAsync returns, so the
  // host plan can be rewritten for the next call right away
  CK(copy_async(h, h->dPlan, &h->hPlan, sizeof(Plan), cudaMemcpyHostToDevice, h->stream));
  return LBM_OK;
}

// Fill the plan's solid set; when `targets` is true also lay out and clear the
// per-sphere impulse arrays.
int set_solids(lbm_sim *h, const lbm_sphere *sp, int ns, bool targets) {
  SolidSet &ss = h->hPlan.ss;
  memset(&ss, 0, sizeof(ss));
  ss.nsph = ns;
  if (h->slab) {
    ss.zlo = h->ownLo;
    ss.zend = h->ownHi + 1;
  }
  long long off = 0;
  int maxChunks = 1;
  long long offs[LBM_MAX_SPHERES] = {0};
  for (int b = 0; b < ns; b++) {
    SphereDesc &d = ss.sph[b];
    d.cx = sp[b].cx;
    d.cy = sp[b].cy;
    // a slab works in its local frame: z - zoff, exactly (cz - zoff is exact
    // for integer zoff, so every contains / surfaceVelocity / torque-arm
    // difference rounds as it does in the global frame)
    d.cz = sp[b].cz - h->zoff;
    d.r = sp[b].r;
    d.vx = sp[b].vx;
    d.vy = sp[b].vy;
    d.vz = sp[b].vz;
    d.wx = sp[b].wx;
    d.wy = sp[b].wy;
    d.wz = sp[b].wz;
    if (!targets) continue;
    Box bx = box_grow(sphere_box(d.cx, d.cy, d.cz, d.r, h->nx, h->ny, h->nz), 1, h->nx, h->ny, h->nz);
    if (h->slab) {  // links of cells outside the owned planes belong to the neighbour
      bx.lo[2] = std::max(bx.lo[2], h->ownLo);
      bx.hi[2] = std::min(bx.hi[2], h->ownHi);
    }
    ImpulseTarget &t = ss.imp[b];
    long long cells = 0;
    if (box_empty(bx)) {
      t.lo[0] = t.lo[1] = t.lo[2] = 0;
      t.dim[0] = t.dim[1] = t.dim[2] = 0;
    } else {
      for (int a = 0; a < 3; a++) {
        t.lo[a] = bx.lo[a];
        t.dim[a] = bx.hi[a] - bx.lo[a] + 1;
      }
      cells = box_cells(bx);
    }
    offs[b] = off;
    off += cells;
    maxChunks = std::max(maxChunks, (int)((cells + RED_CHUNK - 1) / RED_CHUNK));
  }
  h->hPlan.impDoubles = off * 6;
  h->hPlan.redChunks = maxChunks;
  if (!targets) return LBM_OK;
  long long need = std::max(1LL, off * 6);
  if (need > h->impCap) {
    if (h->impAcc) {
      cudaFreeAsync(h->impAcc, h->stream);
      h->deviceBytes -= h->impCap * sizeof(double);
      h->impAcc = nullptr;
    }
    long long cap = need + need / 2;
    DALLOC(h->impAcc, cap * sizeof(double));
    h->impCap = cap;
  }
  long long pneed = (long long)std::max(ns, 1) * maxChunks * 6;
  if (pneed > h->partialsCap) {
    if (h->partials) {
      cudaFreeAsync(h->partials, h->stream);
      h->deviceBytes -= h->partialsCap * sizeof(double);
      h->partials = nullptr;
    }
    DALLOC(h->partials, pneed * sizeof(double));
    h->partialsCap = pneed;
  }
  h->partialsChunks = maxChunks;
  for (int b = 0; b < ns; b++) ss.imp[b].acc = h->impAcc + offs[b] * 6;
  if (off > 0) CK(cudaMemsetAsync(h->impAcc, 0, off * 6 * sizeof(double), h->stream));
  return LBM_OK;
}

int reduce_impulses(lbm_sim *h, double *d_out) {
  int ns = h->hPlan.ss.nsph;
  if (ns == 0) return LBM_OK;
  dim3 g1(h->partialsChunks, ns);
  k_impulse_reduce<<<g1, RED_THREADS, 0, h->stream>>>(&h->dPlan->ss, h->partials, h->partialsChunks, d_out,
                                                      h->redTickets);
  h->launches++;
  CKL("impulse reduction");
  return LBM_OK;
}

int ensure_counts(lbm_sim *h, long long nch) {
  if (nch <= h->countsCap) return LBM_OK;
  if (h->counts) {
    cudaFreeAsync(h->counts, h->stream);
    h->deviceBytes -= h->countsCap * sizeof(int2);
    h->counts = nullptr;
  }
  DALLOC(h->counts, nch * sizeof(int2));
  h->countsCap = nch;
  return LBM_OK;
}

// Launch the fresh / dead compaction over the plan's box U (already on the
// device); maxChunks bounds the plan's chunk count.
int launch_compaction(lbm_sim *h, long long maxChunks) {
  if (maxChunks <= 0) {
    CK(cudaMemsetAsync(h->totals, 0, 2 * sizeof(int), h->stream));
    h->listsValid = true;
    return LBM_OK;
  }
  int rc = ensure_counts(h, maxChunks);
  if (rc) return rc;
  const unsigned ctas = (unsigned)std::min<long long>(maxChunks, SWEEP_CTAS);
  k_compact_count<<<ctas, COMPACT_THREADS, 0, h->stream>>>(h->tag, h->tagPrev, h->nx, h->ny, h->dPlan,
                                                           h->counts);
  k_compact_scan<<<1, 1024, 0, h->stream>>>(h->counts, h->dPlan, h->totals);
  k_compact_emit<<<ctas, COMPACT_THREADS, 0, h->stream>>>(h->tag, h->tagPrev, h->nx, h->ny, h->dPlan,
                                                          h->counts, h->fresh, h->dead, (int)h->listCap);
  h->launches += 3;
  CKL("fresh/dead compaction");
  h->listsValid = true;
  return LBM_OK;
}

// The fused step kernel, bracketed by CUDA events when timing is on.
void launch_fused(lbm_sim *h) {
  if (h->timing) {
    if (h->evUsed == h->evStart.size()) {
      cudaEvent_t a, b;
      cudaEventCreate(&a);
      cudaEventCreate(&b);
      h->evStart.push_back(a);
      h->evStop.push_back(b);
    }
    cudaEventRecord(h->evStart[h->evUsed], h->stream);
    h->ops->fused_step(h, h->cfg);
    cudaEventRecord(h->evStop[h->evUsed], h->stream);
    h->evUsed++;
  } else {
    h->ops->fused_step(h, h->cfg);
  }
}

void set_box(lbm_sim *h, const Box &bx) {
  h->hPlan.U = bx;
  h->hPlan.ucells = box_cells(bx);
  h->hPlan.nchunks = (int)((h->hPlan.ucells + COMPACT_CHUNK - 1) / COMPACT_CHUNK);
}

// fresh / dead lists over a box, scan order
int compact_sets(lbm_sim *h, const Box &bx) {
  set_box(h, bx);
  int rc = upload_plan(h);
  if (rc) return rc;
  return launch_compaction(h, h->hPlan.nchunks);
}

void shift_boxes(lbm_sim *h, const Box &now) {
  h->boxLastLast = h->boxLast;
  h->boxLast = now;
}

// Synchronizes the handle's stream and reports a fused step that was
// abandoned because a bounded wait ran out (LBM_ERR_TIMEOUT; the status is
// cleared, the fields of that step are not valid).  Copies queued before the
// call complete with it.
int sync_status(lbm_sim *h) {
  CK(copy_async(h, h->hTotals + 2, h->totals + 2, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (h->hTotals[2] != 0) {
    h->hTotals[2] = 0;
    CK(cudaMemsetAsync(h->totals + 2, 0, sizeof(int), h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return fail(h, LBM_ERR_TIMEOUT,
                "fused step abandoned: a staged plane did not arrive within the bounded wait");
  }
  return LBM_OK;
}

// NaN/Inf watchdog, opt-in (the reference lets a blow-up show as NaN in the
// fields): once watchEvery steps have completed since the last scan, the
// current phi, rho and u are scanned and a non-finite value fails the call.
int watch_after(lbm_sim *h, long long steps) {
  if (h->watchEvery <= 0) return LBM_OK;
  h->watchSteps += steps;
  if (h->watchSteps < h->watchEvery) return LBM_OK;
  h->watchSteps = 0;
  if (!h->dWatch) DALLOC(h->dWatch, sizeof(unsigned long long));
  CK(cudaMemsetAsync(h->dWatch, 0xFF, sizeof(unsigned long long), h->stream));
  h->ops->watch_finite(h, h->dWatch);
  CKL("NaN watchdog");
  unsigned long long first = 0;
  CK(copy_async(h, &first, h->dWatch, sizeof first, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (first == ~0ull) return LBM_OK;
  const long long i = (long long)first, nxny = (long long)h->nx * h->ny;
  return fail(h, LBM_ERR_NAN,
              "non-finite phi, rho or u at cell " + std::to_string(i) + " (x " + std::to_string(i % h->nx) +
                  ", y " + std::to_string((i / h->nx) % h->ny) + ", z " + std::to_string(i / nxny) + ")");
}

int fetch_out(lbm_sim *h, const double *d_src, int ns, lbm_impulse *out) {
  if (!out || ns == 0) return LBM_OK;
  CK(copy_async(h, h->hOut, d_src, (size_t)ns * 6 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  if (int rc = sync_status(h)) return rc;
  for (int b = 0; b < ns; b++) {
    out[b].Fx = h->hOut[6 * b + 0];
    out[b].Fy = h->hOut[6 * b + 1];
    out[b].Fz = h->hOut[6 * b + 2];
    out[b].Tx = h->hOut[6 * b + 3];
    out[b].Ty = h->hOut[6 * b + 4];
    out[b].Tz = h->hOut[6 * b + 5];
  }
  return LBM_OK;
}

// the sphere fields the dead-cell impulses depend on (set_solids copies
// these; F, T and the mass properties do not enter)
bool same_sphere_geometry(const lbm_sphere &a, const lbm_sphere &b) {
  return a.cx == b.cx && a.cy == b.cy && a.cz == b.cz && a.r == b.r && a.vx == b.vx && a.vy == b.vy &&
         a.vz == b.vz && a.wx == b.wx && a.wy == b.wy && a.wz == b.wz;
}
// record the handle's state with a dead-cell result computed ahead
void dead_ahead_stamp(lbm_sim *h) {
  auto &A = h->deadAhead;
  A.launches = h->launches;
  A.h2d = h->h2dBytes;
  A.d2h = h->d2hBytes;
  A.params = h->params;
  A.cur = h->cur;
}
// the result computed ahead, if nothing has moved since and the spheres are
// the ones it was computed for; consumed either way
bool dead_ahead_take(lbm_sim *h, const lbm_sphere *sp, int ns, lbm_impulse *out) {
  auto &A = h->deadAhead;
  if (!A.valid) return false;
  A.valid = false;
  if (A.ns != ns || A.launches != h->launches || A.h2d != h->h2dBytes || A.d2h != h->d2hBytes ||
      A.cur != h->cur || memcmp(&A.params, &h->params, sizeof(lbm_params)) != 0)
    return false;
  for (int b = 0; b < ns; b++)
    if (!same_sphere_geometry(A.sp[b], sp[b])) return false;
  if (out)
    for (int b = 0; b < ns; b++)
      out[b] = lbm_impulse{A.out[6 * b + 0], A.out[6 * b + 1], A.out[6 * b + 2],
                           A.out[6 * b + 3], A.out[6 * b + 4], A.out[6 * b + 5]};
  return true;
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int now = -1;
    cudaGetDevice(&now);
    if (prev >= 0 && now != prev) cudaSetDevice(prev);
  }
};
// An entry point's guard on one handle: its device, and any dead-cell result
// computed ahead is dropped (the call may move the state it was computed on;
// lbm_step_end computes a new one at its end).
struct EntryGuard : DeviceGuard {
  explicit EntryGuard(lbm_sim *h) : DeviceGuard(h->device) { h->deadAhead.valid = false; }
};

__global__ void k_f32_to_real_d(double *dst, const float *src, long long n) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (double)src[i];
}
__global__ void k_real_d_to_f32(float *dst, const double *src, long long n) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (float)src[i];
}

// float32 host -> device scalar array of the handle's macro type
int put_scalar(lbm_sim *h, void *dst, const float *host) {
  size_t n = (size_t)h->n;
  if (h->ops->macro_bytes() == 4) {
    CK(copy_async(h, dst, host, n * 4, cudaMemcpyHostToDevice, h->stream));
  } else {
    int rc = ensure_staging(h, n * 4);
    if (rc) return rc;
    CK(copy_async(h, h->staging, host, n * 4, cudaMemcpyHostToDevice, h->stream));
    k_f32_to_real_d<<<nblocks(n, 256), 256, 0, h->stream>>>((double *)dst, (const float *)h->staging, n);
    h->launches++;
    CKL("convert");
  }
  return LBM_OK;
}

int get_scalar(lbm_sim *h, const void *src, float *host) {
  size_t n = (size_t)h->n;
  if (h->ops->macro_bytes() == 4) {
    CK(copy_async(h, host, src, n * 4, cudaMemcpyDeviceToHost, h->stream));
  } else {
    int rc = ensure_staging(h, n * 4);
    if (rc) return rc;
    k_real_d_to_f32<<<nblocks(n, 256), 256, 0, h->stream>>>((float *)h->staging, (const double *)src, n);
    h->launches++;
    CKL("convert");
    CK(copy_async(h, host, h->staging, n * 4, cudaMemcpyDeviceToHost, h->stream));
  }
  CK(cudaStreamSynchronize(h->stream));
  return LBM_OK;
}

// device scalar array of the handle's macro type -> double host array
int get_scalar64(lbm_sim *h, const void *src, double *host) {
  size_t n = (size_t)h->n;
  if (h->ops->macro_bytes() == 8) {
    CK(copy_async(h, host, src, n * 8, cudaMemcpyDeviceToHost, h->stream));
  } else {
    int rc = ensure_staging(h, n * 8);
    if (rc) return rc;
    k_f32_to_real_d<<<nblocks(n, 256), 256, 0, h->stream>>>((double *)h->staging, (const float *)src, n);
    h->launches++;
    CKL("convert");
    CK(copy_async(h, host, h->staging, n * 8, cudaMemcpyDeviceToHost, h->stream));
  }
  CK(cudaStreamSynchronize(h->stream));
  return LBM_OK;
}

void free_all(lbm_sim *h) {
  if (h->image) cudaFreeAsync(h->image, h->stream);
  void *ptrs[] = {h->F[0], h->F[1], h->H[0], h->H[1], h->tag, h->tagPrev, h->grad[0], h->grad[1],
                  h->grad[2], h->grad[3], h->us[0], h->us[1], h->us[2], h->bf[0], h->bf[1],
                  h->bf[2], h->fresh, h->dead, h->counts, h->totals, h->impAcc, h->partials,
                  h->dOut, h->dSph, h->staging, h->dPhiCol, h->dPlan, h->dWatch, h->linkChunks,
                  h->linkBuf, h->redTickets, h->meshTri, h->dMaps};
  for (void *p : ptrs)
    if (p) cudaFreeAsync(p, h->stream);
  for (int c = 0; c < 2; c++)
    for (int a = 0; a < 5; a++)
      if (h->mac[c][a]) cudaFreeAsync(h->mac[c][a], h->stream);
  for (cudaEvent_t e : h->evStart) cudaEventDestroy(e);
  for (cudaEvent_t e : h->evStop) cudaEventDestroy(e);
  if (h->hOut) cudaFreeHost(h->hOut);
  if (h->hTotals) cudaFreeHost(h->hTotals);
  if (h->copyStream) cudaStreamSynchronize(h->copyStream);
  for (int b = 0; b < 2; b++) {
    if (h->frameDev[b]) cudaFreeAsync(h->frameDev[b], h->stream);
    if (h->evFrame[b]) cudaEventDestroy(h->evFrame[b]);
    if (h->evPackedSlot[b]) cudaEventDestroy(h->evPackedSlot[b]);
  }
  if (h->evPacked) cudaEventDestroy(h->evPacked);
  if (h->evCopied) cudaEventDestroy(h->evCopied);
  if (h->copyStream) cudaStreamDestroy(h->copyStream);
  if (h->stream) {
    cudaStreamSynchronize(h->stream);  // the stream-ordered frees above
    cudaStreamDestroy(h->stream);
  }
}


// ---------------------------------------------------------------- device-resident coupled step
// One coupled step (sim.step, absorbDeadCells, RigidSphere.step; src/worker.js:96-100)
// entirely on the device: the plan is computed by k_plan from the device sphere
// state, so no host round trip is needed between steps.  Split into the parts a
// batch launches around its shared fused kernel.
struct CoupledCtx {
  int ns = 0;
  long long slotCells = 0, maxU = 0, maxChunks = 0;
  int redChunks = 0;
};

// Capacities for the device-computed plan, the plan's history and the device
// sphere array; everything a captured step needs is allocated here.
int coupled_prepare(lbm_sim *h, const lbm_sphere *sp, int ns, bool frames, CoupledCtx &c) {
  int rc = check_spheres(h, sp, ns);
  if (rc) return rc;
  if (h->slab)
    return fail(h, LBM_ERR_UNSUPPORTED,
                "a z slab steps with lbm_step: its sphere needs every slab's impulses before it moves");
  if (h->bfActive) return fail(h, LBM_ERR_STATE, "a pending body force needs lbm_step");
  if (!h->fusedOK) return fail(h, LBM_ERR_UNSUPPORTED, "grid too large for the fused kernel");
  double rmax = 0;
  for (int b = 0; b < ns; b++) rmax = std::max(rmax, sp[b].r);
  long long side = 2 * (long long)ceil(rmax) + 7;
  c.ns = ns;
  c.slotCells = std::min(h->n, side * side * side);
  long long uside = 2 * (long long)ceil(rmax) + 12;
  c.maxU = (h->fullRetagSteps > 0 || ns > 1) ? h->n : std::min(h->n, uside * uside * uside);
  if (ns == 0) c.maxU = (h->fullRetagSteps > 0) ? h->n : box_cells(box_union(h->boxLast, h->boxLastLast));
  c.maxChunks = (c.maxU + COMPACT_CHUNK - 1) / COMPACT_CHUNK;
  c.redChunks = (int)((c.slotCells + RED_CHUNK - 1) / RED_CHUNK);
  long long need = std::max(1LL, (long long)ns * c.slotCells * 6);
  if (need > h->impCap) {
    if (h->impAcc) {
      cudaFreeAsync(h->impAcc, h->stream);
      h->deviceBytes -= h->impCap * sizeof(double);
      h->impAcc = nullptr;
    }
    DALLOC(h->impAcc, need * sizeof(double));
    h->impCap = need;
  }
  // the slots start at zero; every step's reduction zeroes the slots it reads
  CK(cudaMemsetAsync(h->impAcc, 0, need * sizeof(double), h->stream));
  long long pneed = (long long)std::max(ns, 1) * c.redChunks * 6;
  if (pneed > h->partialsCap) {
    if (h->partials) {
      cudaFreeAsync(h->partials, h->stream);
      h->deviceBytes -= h->partialsCap * sizeof(double);
      h->partials = nullptr;
    }
    DALLOC(h->partials, pneed * sizeof(double));
    h->partialsCap = pneed;
  }
  h->partialsChunks = c.redChunks;
  if ((rc = ensure_counts(h, std::max(1LL, c.maxChunks)))) return rc;
  if (frames && (rc = ensure_staging(h, (size_t)h->n * 2))) return rc;
  // seed the device plan's history from the host's
  memset(&h->hPlan, 0, sizeof(Plan));
  h->hPlan.boxLast = h->boxLast;
  h->hPlan.boxLastLast = h->boxLastLast;
  h->hPlan.fullRetag = h->fullRetagSteps;
  h->hPlan.ss.nsph = ns;
  if ((rc = upload_plan(h))) return rc;
  if (ns > 0)
    CK(copy_async(h, h->dSph, sp, ns * sizeof(lbm_sphere), cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return LBM_OK;
}

// plan, retag, fresh / dead compaction, fresh fill, impulse slot clearing
int coupled_pre(lbm_sim *h, const CoupledCtx &c) {
  k_plan<<<1, 1, 0, h->stream>>>(h->dPlan, h->dSph, c.ns, h->nx, h->ny, h->nz, h->impAcc, c.slotCells,
                                 c.maxU);
  h->launches++;
  h->ops->retag_box(h, c.maxU);
  int rc = launch_compaction(h, c.maxChunks);
  if (rc) return rc;
  h->ops->fresh_fill(h);
  CKL("coupled step (before the fused kernel)");
  return LBM_OK;
}

// impulse reduction, dead-cell absorption, RigidSphere.step on the device
int coupled_post(lbm_sim *h, const CoupledCtx &c) {
  if (c.ns > 0) {
    double *dFluid = h->dOut, *dDead = h->dOut + LBM_MAX_SPHERES * 6;
    dim3 g1(c.redChunks, c.ns);
    k_impulse_reduce<<<g1, RED_THREADS, 0, h->stream>>>(&h->dPlan->ss, h->partials, c.redChunks, dFluid,
                                                        h->redTickets);
    h->ops->absorb_dead(h, dDead);
    h->ops->sphere_step_device(h, h->dSph, c.ns, h->params.gravity, dFluid, dDead);
    h->launches++;
  }
  CKL("coupled step (after the fused kernel)");
  return LBM_OK;
}

// RG8 volume of the current state into host memory dst (pinned when captured);
// fused: the fused step packed planes 1 .. nz-2 into the staging buffer already
int coupled_frame(lbm_sim *h, uint8_t *dst, bool fused = false) {
  if (fused) h->ops->pack_end_planes(h, (uint8_t *)h->staging);
  else h->ops->pack(h, (uint8_t *)h->staging);
  CKL("packVolume");
  CK(copy_async(h, dst, h->staging, (size_t)h->n * 2, cudaMemcpyDeviceToHost, h->stream));
  return LBM_OK;
}

// sphere state and plan history back to the host
int coupled_finish(lbm_sim *h, lbm_sphere *sp, int ns) {
  CK(copy_async(h, &h->hPlan, h->dPlan, sizeof(Plan), cudaMemcpyDeviceToHost, h->stream));
  if (ns > 0)
    CK(copy_async(h, sp, h->dSph, ns * sizeof(lbm_sphere), cudaMemcpyDeviceToHost, h->stream));
  if (int rc = sync_status(h)) return rc;
  h->boxLast = h->hPlan.boxLast;
  h->boxLastLast = h->hPlan.boxLastLast;
  h->fullRetagSteps = h->hPlan.fullRetag;
  h->lastRetagBox = h->hPlan.U;
  h->listsValid = true;
  if (h->hPlan.overflow) return fail(h, LBM_ERR_CAPACITY, "sphere moved beyond the planned retag box");
  return LBM_OK;
}

// the deferred copy of lbm_step_frame's frame, if one is waiting
int flush_frame_copy(lbm_sim *h) {
  if (h->deferredSlot < 0) return LBM_OK;
  const int slot = h->deferredSlot;
  h->deferredSlot = -1;
  CK(cudaStreamWaitEvent(h->copyStream, h->evPackedSlot[slot], 0));
  CK(copy_async(h, h->deferredHost, h->frameDev[slot], (size_t)h->n * 2, cudaMemcpyDeviceToHost, h->copyStream));
  CK(cudaEventRecord(h->evFrame[slot], h->copyStream));
  CK(cudaEventRecord(h->evCopied, h->copyStream));
  h->framePending[slot] = true;
  h->copyPending = true;
  return LBM_OK;
}

// the copy stream, its events and the two device frames of the asynchronous
// frame path, created on first use; *buf receives the frame to pack into, and
// the handle's stream waits until that frame's previous copy is done
int next_frame(lbm_sim *h, uint8_t **buf, int *slot) {
  if (!h->copyStream) {
    CK(cudaStreamCreateWithFlags(&h->copyStream, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&h->evPacked, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&h->evCopied, cudaEventDisableTiming));
  }
  int rc = flush_frame_copy(h);
  if (rc) return rc;
  const int b = h->frameNext;
  if (!h->frameDev[b]) {
    DALLOC(h->frameDev[b], (size_t)h->n * 2);
    CK(cudaEventCreateWithFlags(&h->evFrame[b], cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&h->evPackedSlot[b], cudaEventDisableTiming));
  }
  if (h->framePending[b]) CK(cudaStreamWaitEvent(h->stream, h->evFrame[b], 0));
  *buf = (uint8_t *)h->frameDev[b];
  *slot = b;
  return LBM_OK;
}

// copy the frame packed into buffer `slot` (on the handle's stream) to host
// memory on the copy stream
int issue_frame_copy(lbm_sim *h, int slot, uint8_t *host) {
  CK(cudaEventRecord(h->evPacked, h->stream));
  CK(cudaStreamWaitEvent(h->copyStream, h->evPacked, 0));
  CK(copy_async(h, host, h->frameDev[slot], (size_t)h->n * 2, cudaMemcpyDeviceToHost, h->copyStream));
  CK(cudaEventRecord(h->evFrame[slot], h->copyStream));
  CK(cudaEventRecord(h->evCopied, h->copyStream));
  h->framePending[slot] = true;
  h->copyPending = true;
  h->frameNext = 1 - slot;
  return LBM_OK;
}

}  // namespace

// =====================================================================================
extern "C" {

size_t lbm_footprint_bytes(int nx, int ny, int nz, int storage) {
  if (nx < 3 || ny < 3 || nz < 3 || storage < 0 || storage > 3) return 0;
  long long n = (long long)nx * ny * nz;
  size_t pb = pop_bytes_of(storage), mb = mac_bytes_of(storage);
  size_t bytes = 2 * (size_t)(pop_elems(n, 27) + pop_elems(n, 7)) * pb;  // F, H ping-pong
  bytes += 2 * 5 * (size_t)(n + ARRAY_PAD) * mb;       // macros ping-pong
  bytes += 2 * (size_t)(n + ARRAY_PAD);                // tag, tagPrev
  bytes += 2 * (size_t)n * sizeof(int);                // fresh / dead lists
  return bytes;
}

int lbm_create(int nx, int ny, int nz, int storage, int device, lbm_sim **out) {
  if (!out) return LBM_ERR_ARG;
  *out = nullptr;
  if (nx < 3 || ny < 3 || nz < 3) return LBM_ERR_ARG;
  if ((long long)nx * ny * nz >= (1LL << 31)) return LBM_ERR_ARG;
  OpsBase *ops = ops_for(storage);
  if (!ops) return LBM_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return LBM_ERR_CUDA;
  }
  if (device < 0 || device >= ndev) return LBM_ERR_ARG;
  DeviceGuard g(device);
  lbm_sim *h = new lbm_sim();
  h->nx = nx;
  h->ny = ny;
  h->nz = nz;
  h->storage = storage;
  h->device = device;
  h->ops = ops;
  h->n = (long long)nx * ny * nz;
  h->fusedOK = h->n < (1LL << 31) - 64;  // cell indices are 32-bit in the fused kernel
  // default launch shape: the compact-ring 6-row form with tensor prefetches
  // into L2 (the plain compact form where nx is not a multiple of 16) in
  // z-chunks of 22 planes (FP32) or 24 (FP16, BF16), the fastest measured at
  // 256^3, where the storage form has it (FP32 values in the ring); the
  // plain 4-row form for FP64
  if (ops->shape_ok(6 | LBM_FUSED_L2PF)) {
    h->cfg.ty = 6 | LBM_FUSED_L2PF;
    h->cfg.zchunk = ops->pop_bytes() == 4 ? 22 : 24;
  }
  h->params = lbm_params{0.6, 0.7, 0.012, 0.0010, 1.0, 0.05, 4.0, 0.02};  // src/sim.js:88-95
  int rc = LBM_OK;
  auto body = [&]() -> int {
    keep_pool(device);
    CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    size_t pb = ops->pop_bytes(), mb = ops->macro_bytes();
    for (int c = 0; c < 2; c++) {
      DALLOC(h->F[c], pop_elems(h->n, 27) * pb);
      DALLOC(h->H[c], pop_elems(h->n, 7) * pb);
      CK(cudaMemsetAsync(h->F[c], 0, pop_elems(h->n, 27) * pb, h->stream));
      CK(cudaMemsetAsync(h->H[c], 0, pop_elems(h->n, 7) * pb, h->stream));
      // macro and tag arrays carry a tail pad: the pipelined step copies rows
      // rounded out to 16-byte units, which can reach past the last cell
      for (int a = 0; a < 5; a++) {
        DALLOC(h->mac[c][a], (h->n + ARRAY_PAD) * mb);
        CK(cudaMemsetAsync(h->mac[c][a], 0, (h->n + ARRAY_PAD) * mb, h->stream));
      }
    }
    DALLOC(h->tag, h->n + ARRAY_PAD);
    DALLOC(h->tagPrev, h->n + ARRAY_PAD);
    CK(cudaMemsetAsync(h->tag, 0, h->n + ARRAY_PAD, h->stream));
    CK(cudaMemsetAsync(h->tagPrev, 0, h->n + ARRAY_PAD, h->stream));
    h->listCap = h->n;
    DALLOC(h->fresh, h->listCap * sizeof(int));
    DALLOC(h->dead, h->listCap * sizeof(int));
    DALLOC(h->totals, 3 * sizeof(int));
    CK(cudaMemsetAsync(h->totals, 0, 3 * sizeof(int), h->stream));
    DALLOC(h->dOut, 2 * LBM_MAX_SPHERES * 6 * sizeof(double));
    DALLOC(h->redTickets, LBM_MAX_SPHERES * sizeof(unsigned));
    CK(cudaMemsetAsync(h->redTickets, 0, LBM_MAX_SPHERES * sizeof(unsigned), h->stream));
    DALLOC(h->dSph, LBM_MAX_SPHERES * sizeof(lbm_sphere));
    DALLOC(h->dPlan, sizeof(Plan));
    CK(cudaMemsetAsync(h->dPlan, 0, sizeof(Plan), h->stream));
    DALLOC(h->dPhiCol, (size_t)ny * sizeof(double));
    CK(cudaMallocHost((void **)&h->hOut, 2 * LBM_MAX_SPHERES * 6 * sizeof(double)));
    CK(cudaMallocHost((void **)&h->hTotals, 3 * sizeof(int)));
    CK(cudaStreamSynchronize(h->stream));
    return LBM_OK;
  };
  rc = body();
  if (rc == LBM_OK) rc = ops->build_stage_maps(h);
  if (rc != LBM_OK) {
    free_all(h);
    delete h;
    return rc;
  }
  // A fresh Sim has every cell FLUID (zeroed Uint8Array); the first retag
  // covers the whole grid so the walls get their tags.
  h->fullRetagSteps = 2;
  *out = h;
  return LBM_OK;
}

int lbm_destroy(lbm_sim *h) {
  if (!h) return LBM_ERR_ARG;
  EntryGuard g(h);
  if (h->stream) cudaStreamSynchronize(h->stream);
  free_all(h);
  delete h;
  return LBM_OK;
}

const char *lbm_last_error(const lbm_sim *h) { return h ? h->err.c_str() : "null handle"; }

int lbm_get_dims(const lbm_sim *h, int *nx, int *ny, int *nz, int *storage) {
  if (!h) return LBM_ERR_ARG;
  if (nx) *nx = h->nx;
  if (ny) *ny = h->ny;
  if (nz) *nz = h->nz;
  if (storage) *storage = h->storage;
  return LBM_OK;
}

int lbm_device_bytes(const lbm_sim *h, size_t *bytes) {
  if (!h || !bytes) return LBM_ERR_ARG;
  *bytes = h->deviceBytes;
  return LBM_OK;
}

int lbm_set_params(lbm_sim *h, const lbm_params *p) {
  if (!h || !p) return fail(h, LBM_ERR_ARG, "null");
  h->params = *p;
  return LBM_OK;
}

int lbm_get_params(const lbm_sim *h, lbm_params *p) {
  if (!h || !p) return LBM_ERR_ARG;
  *p = h->params;
  return LBM_OK;
}

static size_t field_count(const lbm_sim *h, int field) {
  if (field == LBM_FIELD_F || field == LBM_FIELD_F2) return (size_t)h->n * 27;
  if (field == LBM_FIELD_H || field == LBM_FIELD_H2) return (size_t)h->n * 7;
  return (size_t)h->n;
}

static int pops_transfer(lbm_sim *h, int field, const float *up, float *down) {
  bool isH = field == LBM_FIELD_H || field == LBM_FIELD_H2;
  bool second = field == LBM_FIELD_F2 || field == LBM_FIELD_H2;
  int Q = isH ? 7 : 27;
  long long chunk = std::min<long long>(h->n, 1 << 20);
  int rc = ensure_staging(h, (size_t)chunk * Q * sizeof(float));
  if (rc) return rc;
  for (long long c0 = 0; c0 < h->n; c0 += chunk) {
    long long cells = std::min(chunk, h->n - c0);
    if (up) {
      CK(copy_async(h, h->staging, up + c0 * Q, cells * Q * sizeof(float), cudaMemcpyHostToDevice,
                         h->stream));
      h->ops->upload_pops(h, isH, second ? 2 : 0, (const float *)h->staging, c0, cells);
      CKL("upload populations");
      CK(cudaStreamSynchronize(h->stream));
    } else {
      h->ops->download_pops(h, isH, second ? 2 : 1, (float *)h->staging, c0, cells);
      CKL("download populations");
      CK(copy_async(h, down + c0 * Q, h->staging, cells * Q * sizeof(float), cudaMemcpyDeviceToHost,
                         h->stream));
      CK(cudaStreamSynchronize(h->stream));
    }
  }
  return LBM_OK;
}

int lbm_upload_field(lbm_sim *h, int field, const void *host, size_t count) {
  if (!h || !host) return fail(h, LBM_ERR_ARG, "null");
  if (field < 0 || field >= LBM_FIELD_COUNT) return fail(h, LBM_ERR_ARG, "unknown field");
  if (count != field_count(h, field)) return fail(h, LBM_ERR_ARG, "element count mismatch");
  EntryGuard g(h);
  const float *src = (const float *)host;
  size_t n = (size_t)h->n;
  switch (field) {
    case LBM_FIELD_F:
    case LBM_FIELD_F2:
    case LBM_FIELD_H:
    case LBM_FIELD_H2:
      return pops_transfer(h, field, src, nullptr);
    case LBM_FIELD_TAG:
    case LBM_FIELD_TAG_PREV:
      CK(copy_async(h, field == LBM_FIELD_TAG ? h->tag : h->tagPrev, host, n, cudaMemcpyHostToDevice,
                         h->stream));
      CK(cudaStreamSynchronize(h->stream));
      h->fullRetagSteps = 2;
      h->listsValid = false;
      return LBM_OK;
    case LBM_FIELD_PHI_PREV:
      // phiPrev is overwritten from phi by the next retagCells before anything
      // reads it (src/sim.js:216-217); a write to it has no effect on the run.
      return LBM_OK;
    case LBM_FIELD_PHI: {
      size_t mb = h->ops->macro_bytes();
      void *old = nullptr;
      bool off = !h->ops->phases_supported();
      if (off) {
        CK(cudaMallocAsync(&old, n * mb, h->stream));
      }
      for (int c = 0; c < 2; c++) {
        if (off) CK(copy_async(h, old, h->mac[c][0], n * mb, cudaMemcpyDeviceToDevice, h->stream));
        int rc = put_scalar(h, h->mac[c][0], src);
        if (rc) {
          if (old) cudaFreeAsync(old, h->stream);
          return rc;
        }
        if (off) h->ops->reencode_h(h, c, old);
      }
      if (old) cudaFreeAsync(old, h->stream);
      cudaError_t e = cudaStreamSynchronize(h->stream);
      if (e != cudaSuccess) return cuda_fail(h, "upload phi", e);
      return LBM_OK;
    }
    case LBM_FIELD_RHO:
    case LBM_FIELD_UX:
    case LBM_FIELD_UY:
    case LBM_FIELD_UZ: {
      int a = field - LBM_FIELD_RHO + 1;
      const bool pad = (field == LBM_FIELD_UX || field == LBM_FIELD_UY) && h->ops->u_in_pads();
      for (int c = 0; c < 2; c++) {
        int rc = put_scalar(h, h->mac[c][a], src);
        if (rc) return rc;
        if (pad) h->ops->u_array(h, field - LBM_FIELD_UX, c, h->mac[c][a], true);
      }
      CKL("upload u");
      CK(cudaStreamSynchronize(h->stream));
      return LBM_OK;
    }
    default: {
      void **arr = nullptr;
      if (field >= LBM_FIELD_USX && field <= LBM_FIELD_USZ) arr = &h->us[field - LBM_FIELD_USX];
      else if (field >= LBM_FIELD_GX && field <= LBM_FIELD_LAP) arr = &h->grad[field - LBM_FIELD_GX];
      else arr = &h->bf[field - LBM_FIELD_BODY_FX];
      int rc = ensure_scalar(h, arr);
      if (rc) return rc;
      rc = put_scalar(h, *arr, src);
      if (rc) return rc;
      if (field >= LBM_FIELD_BODY_FX) {
        for (int a = 0; a < 3; a++) {
          rc = ensure_scalar(h, &h->bf[a]);
          if (rc) return rc;
        }
        h->bfActive = true;
      }
      CK(cudaStreamSynchronize(h->stream));
      return LBM_OK;
    }
  }
}

int lbm_download_field(lbm_sim *h, int field, void *host, size_t count) {
  if (!h || !host) return fail(h, LBM_ERR_ARG, "null");
  if (field < 0 || field >= LBM_FIELD_COUNT) return fail(h, LBM_ERR_ARG, "unknown field");
  if (count != field_count(h, field)) return fail(h, LBM_ERR_ARG, "element count mismatch");
  EntryGuard g(h);
  float *dst = (float *)host;
  size_t n = (size_t)h->n;
  switch (field) {
    case LBM_FIELD_F:
    case LBM_FIELD_F2:
    case LBM_FIELD_H:
    case LBM_FIELD_H2:
      return pops_transfer(h, field, nullptr, dst);
    case LBM_FIELD_TAG:
    case LBM_FIELD_TAG_PREV:
      CK(copy_async(h, host, field == LBM_FIELD_TAG ? h->tag : h->tagPrev, n, cudaMemcpyDeviceToHost,
                         h->stream));
      CK(cudaStreamSynchronize(h->stream));
      return LBM_OK;
    case LBM_FIELD_PHI_PREV:
      return get_scalar(h, h->mac[1 - h->cur][0], dst);
    case LBM_FIELD_PHI:
    case LBM_FIELD_RHO:
    case LBM_FIELD_UX:
    case LBM_FIELD_UY:
    case LBM_FIELD_UZ:
      // macro slots: 0 phi, 1 rho, 2 ux, 3 uy, 4 uz (ux, uy gathered first
      // from the population pads where the storage form keeps them there)
      if ((field == LBM_FIELD_UX || field == LBM_FIELD_UY) && h->ops->u_in_pads()) {
        h->ops->u_array(h, field - LBM_FIELD_UX, h->cur, h->mac[h->cur][field - LBM_FIELD_RHO + 1], false);
        CKL("download u");
      }
      return get_scalar(h, h->mac[h->cur][field == LBM_FIELD_PHI ? 0 : field - LBM_FIELD_RHO + 1], dst);
    default: {
      void *arr = nullptr;
      if (field >= LBM_FIELD_USX && field <= LBM_FIELD_USZ) arr = h->us[field - LBM_FIELD_USX];
      else if (field >= LBM_FIELD_GX && field <= LBM_FIELD_LAP) arr = h->grad[field - LBM_FIELD_GX];
      else arr = h->bf[field - LBM_FIELD_BODY_FX];
      if (!arr) {
        memset(dst, 0, n * sizeof(float));
        return LBM_OK;
      }
      return get_scalar(h, arr, dst);
    }
  }
}

int lbm_download_field_f64(lbm_sim *h, int field, double *host, size_t count) {
  if (!h || !host) return fail(h, LBM_ERR_ARG, "null");
  if (field < 0 || field >= LBM_FIELD_COUNT) return fail(h, LBM_ERR_ARG, "unknown field");
  if (field == LBM_FIELD_TAG || field == LBM_FIELD_TAG_PREV)
    return fail(h, LBM_ERR_ARG, "tags are uint8; use lbm_download_field");
  if (count != field_count(h, field)) return fail(h, LBM_ERR_ARG, "element count mismatch");
  EntryGuard g(h);
  size_t n = (size_t)h->n;
  if (field <= LBM_FIELD_H2) {
    bool isH = field == LBM_FIELD_H || field == LBM_FIELD_H2;
    bool second = field == LBM_FIELD_F2 || field == LBM_FIELD_H2;
    int Q = isH ? 7 : 27;
    long long chunk = std::min<long long>(h->n, 1 << 19);
    int rc = ensure_staging(h, (size_t)chunk * Q * sizeof(double));
    if (rc) return rc;
    for (long long c0 = 0; c0 < h->n; c0 += chunk) {
      long long cells = std::min(chunk, h->n - c0);
      h->ops->download_pops64(h, isH, second ? 2 : 1, (double *)h->staging, c0, cells);
      CKL("download populations");
      CK(copy_async(h, host + c0 * Q, h->staging, cells * Q * sizeof(double), cudaMemcpyDeviceToHost,
                    h->stream));
      CK(cudaStreamSynchronize(h->stream));
    }
    return LBM_OK;
  }
  const void *arr = nullptr;
  if ((field == LBM_FIELD_UX || field == LBM_FIELD_UY) && h->ops->u_in_pads()) {
    h->ops->u_array(h, field - LBM_FIELD_UX, h->cur, h->mac[h->cur][field - LBM_FIELD_RHO + 1], false);
    CKL("download u");
  }
  if (field == LBM_FIELD_PHI_PREV) arr = h->mac[1 - h->cur][0];
  else if (field >= LBM_FIELD_RHO && field <= LBM_FIELD_PHI)
    arr = h->mac[h->cur][field == LBM_FIELD_PHI ? 0 : field - LBM_FIELD_RHO + 1];
  else if (field >= LBM_FIELD_USX && field <= LBM_FIELD_USZ) arr = h->us[field - LBM_FIELD_USX];
  else if (field >= LBM_FIELD_GX && field <= LBM_FIELD_LAP) arr = h->grad[field - LBM_FIELD_GX];
  else arr = h->bf[field - LBM_FIELD_BODY_FX];
  if (!arr) {
    memset(host, 0, n * sizeof(double));
    return LBM_OK;
  }
  return get_scalar64(h, arr, host);
}

int lbm_init_flat(lbm_sim *h, double waterlineY) {
  if (!h) return LBM_ERR_ARG;
  EntryGuard g(h);
  std::vector<double> col(h->ny);
  for (int y = 0; y < h->ny; y++) col[y] = 0.5 * (1 + tanh(2 * ((double)y - waterlineY) / h->params.W));
  CK(copy_async(h, h->dPhiCol, col.data(), h->ny * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  h->ops->init_flat(h, h->dPhiCol);
  CKL("init_flat");
  h->ops->seed_hydrostatic(h);
  CKL("seed_hydrostatic");
  CK(cudaStreamSynchronize(h->stream));
  h->boxLast = h->boxLastLast = Box{{1, 1, 1}, {0, 0, 0}};
  h->fullRetagSteps = 0;
  h->listsValid = false;
  return LBM_OK;
}

int lbm_init_profile(lbm_sim *h, const double *phi_col, int ny) {
  if (!h || !phi_col || ny != h->ny) return LBM_ERR_ARG;
  EntryGuard g(h);
  CK(copy_async(h, h->dPhiCol, phi_col, h->ny * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  h->ops->init_flat(h, h->dPhiCol);
  CKL("init_profile");
  h->ops->seed_hydrostatic(h);
  CKL("seed_hydrostatic");
  CK(cudaStreamSynchronize(h->stream));
  h->boxLast = h->boxLastLast = Box{{1, 1, 1}, {0, 0, 0}};
  h->fullRetagSteps = 0;
  h->listsValid = false;
  return LBM_OK;
}

int lbm_seed_hydrostatic(lbm_sim *h) {
  if (!h) return LBM_ERR_ARG;
  EntryGuard g(h);
  h->ops->seed_hydrostatic(h);
  CKL("seed_hydrostatic");
  CK(cudaStreamSynchronize(h->stream));
  return LBM_OK;
}

static int need_phases(lbm_sim *h) {
  if (!h->ops->phases_supported())
    return fail(h, LBM_ERR_UNSUPPORTED,
                "phase-by-phase entry points need FP32 or FP64 storage; FP16/BF16 run lbm_step only");
  return ensure_phase_scratch(h);
}

int lbm_retag_cells(lbm_sim *h, const lbm_sphere *sp, int ns) {
  if (!h) return LBM_ERR_ARG;
  int rc = check_spheres(h, sp, ns);
  if (rc) return rc;
  EntryGuard g(h);
  if ((rc = need_phases(h))) return rc;
  if ((rc = set_solids(h, sp, ns, false))) return rc;
  if ((rc = upload_plan(h))) return rc;
  h->ops->retag_full(h);
  CKL("retag");
  shift_boxes(h, spheres_box(h, sp, ns));
  h->lastRetagBox = interior(h);
  h->fullRetagSteps = h->fullRetagSteps > 0 ? h->fullRetagSteps - 1 : 0;
  h->listsValid = false;
  return LBM_OK;
}

int lbm_retag_cells_mask(lbm_sim *h, const uint8_t *solid_mask, const float *surface_velocity) {
  if (!h || !solid_mask) return LBM_ERR_ARG;
  EntryGuard g(h);
  int rc = need_phases(h);
  if (rc) return rc;
  const size_t n = (size_t)h->n;
  const size_t usOff = (n + 255) / 256 * 256;
  if ((rc = ensure_staging(h, usOff + (surface_velocity ? 12 * n : 0)))) return rc;
  uint8_t *dMask = (uint8_t *)h->staging;
  float *dUs = surface_velocity ? (float *)((uint8_t *)h->staging + usOff) : nullptr;
  CK(copy_async(h, dMask, solid_mask, n, cudaMemcpyHostToDevice, h->stream));
  if (dUs) CK(copy_async(h, dUs, surface_velocity, 12 * n, cudaMemcpyHostToDevice, h->stream));
  h->ops->retag_mask(h, dMask, dUs);
  CKL("retag (mask)");
  CK(cudaStreamSynchronize(h->stream));  // the staging buffer is reused by the next call
  // solid cells may be anywhere: a following fused step retags the whole grid
  h->fullRetagSteps = 2;
  h->lastRetagBox = interior(h);
  h->listsValid = false;
  return LBM_OK;
}

// a mesh's cells and surface velocity into the staging buffer (mask at 0, the
// velocities at *usOff): the whole grid cleared, the mesh's bounding box
// grown by one cell voxelised
static int voxelize_mesh(lbm_sim *h, const double *tri, int ntri, const lbm_rigid_motion *m, size_t *usOff) {
  const size_t n = (size_t)h->n;
  *usOff = (n + 255) / 256 * 256;
  int rc = ensure_staging(h, *usOff + 12 * n);
  if (rc) return rc;
  uint8_t *dMask = (uint8_t *)h->staging;
  float *dUs = (float *)((uint8_t *)h->staging + *usOff);
  CK(cudaMemsetAsync(dMask, 0, n, h->stream));
  CK(cudaMemsetAsync(dUs, 0, 12 * n, h->stream));
  if (ntri == 0) return LBM_OK;
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (long long j = 0; j < 3LL * ntri; j++)
    for (int a = 0; a < 3; a++) {
      const double v = tri[3 * j + a];
      if (!(v == v)) return fail(h, LBM_ERR_ARG, "mesh vertex is NaN");
      lo[a] = std::min(lo[a], v);
      hi[a] = std::max(hi[a], v);
    }
  const int dimsN[3] = {h->nx, h->ny, h->nz};
  int b0[3], b1[3];
  for (int a = 0; a < 3; a++) {
    b0[a] = (int)std::max(0.0, std::floor(lo[a]) - 1.0);
    b1[a] = (int)std::min((double)dimsN[a] - 1, std::ceil(hi[a]) + 1.0);
    if (b1[a] < b0[a]) return LBM_OK;  // the mesh lies outside the grid
  }
  const size_t tb = (size_t)ntri * 9 * sizeof(double);
  if (tb > h->meshCap) {
    if (h->meshTri) {
      cudaFreeAsync(h->meshTri, h->stream);
      h->deviceBytes -= h->meshCap;
      h->meshTri = nullptr;
    }
    DALLOC(h->meshTri, tb);
    h->meshCap = tb;
  }
  CK(copy_async(h, h->meshTri, tri, tb, cudaMemcpyHostToDevice, h->stream));
  const int3 lo3 = make_int3(b0[0], b0[1], b0[2]);
  const int3 dim3_ = make_int3(b1[0] - b0[0] + 1, b1[1] - b0[1] + 1, b1[2] - b0[2] + 1);
  const long long cells = (long long)dim3_.x * dim3_.y * dim3_.z;
  MeshMotion mm{m->cx, m->cy, m->cz, m->vx, m->vy, m->vz, m->wx, m->wy, m->wz};
  k_voxelize_mesh<<<nblocks(cells, MESH_THREADS), MESH_THREADS, 0, h->stream>>>(
      (const double *)h->meshTri, ntri, h->nx, h->ny, lo3, dim3_, mm, dMask, dUs);
  h->launches++;
  CKL("voxelize mesh");
  return LBM_OK;
}

int lbm_voxelize_mesh(lbm_sim *h, const double *tri, int ntri, const lbm_rigid_motion *m, uint8_t *mask_out,
                      float *us_out) {
  if (!h || ntri < 0 || (ntri > 0 && !tri) || !m || !mask_out) return LBM_ERR_ARG;
  EntryGuard g(h);
  size_t usOff = 0;
  int rc = voxelize_mesh(h, tri, ntri, m, &usOff);
  if (rc) return rc;
  CK(copy_async(h, mask_out, h->staging, (size_t)h->n, cudaMemcpyDeviceToHost, h->stream));
  if (us_out)
    CK(copy_async(h, us_out, (uint8_t *)h->staging + usOff, 12 * (size_t)h->n, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return LBM_OK;
}

int lbm_retag_cells_mesh(lbm_sim *h, const double *tri, int ntri, const lbm_rigid_motion *m) {
  if (!h || ntri < 0 || (ntri > 0 && !tri) || !m) return LBM_ERR_ARG;
  EntryGuard g(h);
  int rc = need_phases(h);
  if (rc) return rc;
  size_t usOff = 0;
  if ((rc = voxelize_mesh(h, tri, ntri, m, &usOff))) return rc;
  h->ops->retag_mask(h, (const uint8_t *)h->staging, (const float *)((uint8_t *)h->staging + usOff));
  CKL("retag (mesh)");
  CK(cudaStreamSynchronize(h->stream));  // the staging buffer is reused by the next call
  h->fullRetagSteps = 2;
  h->lastRetagBox = interior(h);
  h->listsValid = false;
  return LBM_OK;
}

int lbm_solid_links(lbm_sim *h, int32_t *cells, int8_t *dirs, double *mom, int cap, int *count) {
  if (!h || !count || cap < 0 || (cap > 0 && (!cells || !dirs || !mom))) return LBM_ERR_ARG;
  EntryGuard g(h);
  int rc = need_phases(h);
  if (rc) return rc;
  const long long chunks = (h->n + LINK_CHUNK - 1) / LINK_CHUNK;
  if (chunks + 1 > h->linkChunksCap) {
    if (h->linkChunks) {
      cudaFreeAsync(h->linkChunks, h->stream);
      h->deviceBytes -= h->linkChunksCap * sizeof(int);
      h->linkChunks = nullptr;
    }
    DALLOC(h->linkChunks, (chunks + 1) * sizeof(int));
    h->linkChunksCap = chunks + 1;
  }
  h->ops->link_count(h, h->linkChunks);
  CKL("link count");
  CK(copy_async(h, h->hTotals, h->linkChunks + chunks, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  const int total = h->hTotals[0];
  *count = total;
  if (cap == 0 || total == 0) return LBM_OK;
  const int take = std::min(cap, total);
  const long long per = sizeof(double) + sizeof(int) + 1;
  if (take > h->linkBufCap) {
    if (h->linkBuf) {
      cudaFreeAsync(h->linkBuf, h->stream);
      h->deviceBytes -= h->linkBufCap * per;
      h->linkBuf = nullptr;
    }
    DALLOC(h->linkBuf, (size_t)take * per);
    h->linkBufCap = take;
  }
  double *dMom = (double *)h->linkBuf;
  int *dCells = (int *)(dMom + h->linkBufCap);
  int8_t *dDirs = (int8_t *)(dCells + h->linkBufCap);
  h->ops->link_emit(h, h->linkChunks, take, dCells, dDirs, dMom);
  CKL("link emit");
  CK(copy_async(h, cells, dCells, (size_t)take * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(copy_async(h, dirs, dDirs, (size_t)take, cudaMemcpyDeviceToHost, h->stream));
  CK(copy_async(h, mom, dMom, (size_t)take * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return LBM_OK;
}

int lbm_handle_fresh_cells(lbm_sim *h) {
  if (!h) return LBM_ERR_ARG;
  EntryGuard g(h);
  int rc = need_phases(h);
  if (rc) return rc;
  if ((rc = compact_sets(h, h->lastRetagBox))) return rc;
  h->ops->fresh_fill(h);
  CKL("fresh cells");
  return LBM_OK;
}

int lbm_compute_phi_gradients(lbm_sim *h) {
  if (!h) return LBM_ERR_ARG;
  EntryGuard g(h);
  int rc = need_phases(h);
  if (rc) return rc;
  h->ops->gradients(h);
  CKL("gradients");
  return LBM_OK;
}

int lbm_collide_phase(lbm_sim *h) {
  if (!h) return LBM_ERR_ARG;
  EntryGuard g(h);
  int rc = need_phases(h);
  if (rc) return rc;
  h->ops->collide_phase(h);
  CKL("collidePhase");
  return LBM_OK;
}

int lbm_stream_phase(lbm_sim *h) {
  if (!h) return LBM_ERR_ARG;
  EntryGuard g(h);
  int rc = need_phases(h);
  if (rc) return rc;
  h->ops->stream_phase(h);
  CKL("streamPhase");
  return LBM_OK;
}

int lbm_collide_hydro(lbm_sim *h) {
  if (!h) return LBM_ERR_ARG;
  EntryGuard g(h);
  int rc = need_phases(h);
  if (rc) return rc;
  h->ops->collide_hydro(h);
  CKL("collideHydro");
  return LBM_OK;
}

int lbm_stream_hydro_and_macro(lbm_sim *h, const lbm_sphere *sp, int ns, lbm_impulse *out) {
  if (!h) return LBM_ERR_ARG;
  int rc = check_spheres(h, sp, ns);
  if (rc) return rc;
  EntryGuard g(h);
  if ((rc = need_phases(h))) return rc;
  if ((rc = set_solids(h, sp, ns, true))) return rc;
  if ((rc = upload_plan(h))) return rc;
  h->ops->stream_hydro_macro(h);
  CKL("streamHydroAndMacro");
  if (h->bfActive) {  // bodyF.fill(0) (src/sim.js:581)
    for (int a = 0; a < 3; a++) CK(cudaMemsetAsync(h->bf[a], 0, h->n * h->ops->macro_bytes(), h->stream));
    h->bfActive = false;
  }
  if ((rc = reduce_impulses(h, h->dOut))) return rc;
  if ((rc = fetch_out(h, h->dOut, ns, out))) return rc;
  return watch_after(h, 1);
}

int lbm_step_begin(lbm_sim *h, const lbm_sphere *sp, int ns) {
  if (!h) return LBM_ERR_ARG;
  int rc = check_spheres(h, sp, ns);
  if (rc) return rc;
  if (h->stepBegunNs >= 0) return fail(h, LBM_ERR_STATE, "a step was begun and not ended");
  EntryGuard g(h);
  if (h->bfActive || !h->fusedOK) {
    // A pending external body force is consumed by the phase-by-phase path,
    // which reads it (src/sim.js:434-436, 558-560); grids too large for the
    // fused kernel's 32-bit indexing take the same path.
    if ((rc = lbm_retag_cells(h, sp, ns))) return rc;
    if ((rc = lbm_handle_fresh_cells(h))) return rc;
    h->stepBegunNs = ns;
    return LBM_OK;
  }
  if ((rc = set_solids(h, sp, ns, true))) return rc;
  Box now = spheres_box(h, sp, ns);
  Box U;
  if (h->fullRetagSteps > 0) {
    U = Box{{0, 0, 0}, {h->nx - 1, h->ny - 1, h->nz - 1}};
    h->fullRetagSteps--;
  } else {
    U = box_union(box_union(now, h->boxLast), h->boxLastLast);
  }
  set_box(h, U);
  h->hPlan.boxLast = h->boxLast;
  h->hPlan.boxLastLast = h->boxLastLast;
  if ((rc = upload_plan(h))) return rc;
  h->ops->retag_box(h, h->hPlan.ucells);
  CKL("retag box");
  h->lastRetagBox = U;
  if ((rc = launch_compaction(h, h->hPlan.nchunks))) return rc;
  h->ops->fresh_fill(h);
  CKL("fresh cells");
  h->stepNow = now;
  h->stepBegunNs = ns;
  return LBM_OK;
}

int lbm_step_end(lbm_sim *h, const lbm_sphere *sp, int ns, lbm_impulse *out) {
  if (!h) return LBM_ERR_ARG;
  int rc = check_spheres(h, sp, ns);
  if (rc) return rc;
  if (h->stepBegunNs < 0) return fail(h, LBM_ERR_STATE, "lbm_step_end without lbm_step_begin");
  if (ns != h->stepBegunNs) return fail(h, LBM_ERR_ARG, "lbm_step_end with another sphere count than its begin");
  h->stepBegunNs = -1;
  EntryGuard g(h);
  if (h->bfActive || !h->fusedOK) {
    if ((rc = lbm_compute_phi_gradients(h))) return rc;
    if ((rc = lbm_collide_phase(h))) return rc;
    if ((rc = lbm_stream_phase(h))) return rc;
    if ((rc = lbm_collide_hydro(h))) return rc;
    return lbm_stream_hydro_and_macro(h, sp, ns, out);
  }
  launch_fused(h);
  CKL("fused step");
  if ((rc = flush_frame_copy(h))) return rc;
  if ((rc = reduce_impulses(h, h->dOut))) return rc;
  h->cur = 1 - h->cur;
  shift_boxes(h, h->stepNow);
  h->deadAhead.valid = false;
  if (ns > 0 && out && h->listsValid) {
    // absorbDeadCells follows every step (src/worker.js:96-100) and reads
    // only the new half and this step's dead list with the same spheres:
    // run it now on the step's plan and fetch it with the step's impulses,
    // so lbm_absorb_dead_cells needs no launch and no wait of its own
    double *d = h->dOut + LBM_MAX_SPHERES * 6;
    h->ops->absorb_dead(h, d);
    CKL("absorbDeadCells");
    CK(copy_async(h, h->hOut + LBM_MAX_SPHERES * 6, d, (size_t)ns * 6 * sizeof(double), cudaMemcpyDeviceToHost,
                  h->stream));
    if ((rc = fetch_out(h, h->dOut, ns, out))) return rc;
    auto &A = h->deadAhead;
    A.ns = ns;
    memcpy(A.sp, sp, (size_t)ns * sizeof(lbm_sphere));
    memcpy(A.out, h->hOut + LBM_MAX_SPHERES * 6, (size_t)ns * 6 * sizeof(double));
    A.valid = true;
  } else if ((rc = fetch_out(h, h->dOut, ns, out))) {
    return rc;
  }
  rc = watch_after(h, 1);
  if (h->deadAhead.valid) dead_ahead_stamp(h);  // the watchdog's scan moves nothing
  return rc;
}

int lbm_step(lbm_sim *h, const lbm_sphere *sp, int ns, lbm_impulse *out) {
  int rc = lbm_step_begin(h, sp, ns);
  if (rc) return rc;
  return lbm_step_end(h, sp, ns, out);
}

int lbm_step_frame(lbm_sim *h, const lbm_sphere *sp, int ns, lbm_impulse *out, uint8_t *host_frame) {
  if (!h || !host_frame) return LBM_ERR_ARG;
  if (h->bfActive || !h->fusedOK) {
    int rc = lbm_step(h, sp, ns, out);
    return rc ? rc : lbm_pack_volume_async(h, host_frame);
  }
  EntryGuard g(h);
  int rc = lbm_step_begin(h, sp, ns);
  if (rc) return rc;
  uint8_t *buf = nullptr;
  int slot = 0;
  if ((rc = next_frame(h, &buf, &slot))) {
    h->stepBegunNs = -1;
    return rc;
  }
  h->fusePack = buf;
  rc = lbm_step_end(h, sp, ns, out);
  h->fusePack = nullptr;
  if (rc && rc != LBM_ERR_NAN) return rc;
  const int stepRc = rc;
  h->ops->pack_end_planes(h, buf);
  CKL("packVolume (end planes)");
  if (h->deadAhead.valid) dead_ahead_stamp(h);  // the pack writes the frame only
  // the copy to the host is issued with the next step's fused kernel (or by
  // any wait for frames), so the step's own small read-backs do not queue
  // behind it on the copy engine
  CK(cudaEventRecord(h->evPackedSlot[slot], h->stream));
  h->deferredSlot = slot;
  h->deferredHost = host_frame;
  h->frameNext = 1 - slot;
  return stepRc;
}

int lbm_absorb_dead_cells(lbm_sim *h, const lbm_sphere *sp, int ns, lbm_impulse *out) {
  if (!h) return LBM_ERR_ARG;
  int rc = check_spheres(h, sp, ns);
  if (rc) return rc;
  if (ns == 0) return LBM_OK;
  if (dead_ahead_take(h, sp, ns, out)) return LBM_OK;
  EntryGuard g(h);
  if (!h->listsValid && (rc = compact_sets(h, h->lastRetagBox))) return rc;
  if ((rc = set_solids(h, sp, ns, false))) return rc;
  if ((rc = upload_plan(h))) return rc;
  double *d = h->dOut + LBM_MAX_SPHERES * 6;
  h->ops->absorb_dead(h, d);
  CKL("absorbDeadCells");
  return fetch_out(h, d, ns, out);
}

int lbm_pack_volume_device(lbm_sim *h, void *dev_out) {
  if (!h || !dev_out) return fail(h, LBM_ERR_ARG, "null");
  EntryGuard g(h);
  h->ops->pack(h, (uint8_t *)dev_out);
  CKL("packVolume");
  return LBM_OK;
}

int lbm_prepare_device(int device, int storage, uint64_t reserve_bytes) {
  OpsBase *ops = ops_for(storage);
  int ndev = 0;
  if (!ops || cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return LBM_ERR_ARG;
  }
  DeviceGuard g(device);
  keep_pool(device);
  ops->warm(device);
  if (reserve_bytes == 0) return LBM_OK;
  // one allocation of the reserve, freed again: the pool keeps its memory
  cudaStream_t st = nullptr;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    return LBM_ERR_CUDA;
  }
  int rc = LBM_OK;
  void *p = nullptr;
  if (cudaMallocAsync(&p, (size_t)reserve_bytes, st) != cudaSuccess) {
    cudaGetLastError();
    rc = LBM_ERR_OOM;
  } else if (cudaFreeAsync(p, st) != cudaSuccess) {
    rc = LBM_ERR_CUDA;
  }
  if (cudaStreamSynchronize(st) != cudaSuccess && rc == LBM_OK) rc = LBM_ERR_CUDA;
  cudaStreamDestroy(st);
  cudaGetLastError();
  return rc;
}

int lbm_trim_device_memory(int device) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return LBM_ERR_ARG;
  }
  DeviceGuard g(device);
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) != cudaSuccess) {
    cudaGetLastError();
    return LBM_ERR_CUDA;
  }
  return cudaMemPoolTrimTo(pool, 0) == cudaSuccess ? LBM_OK : LBM_ERR_CUDA;
}

int lbm_host_alloc(size_t bytes, void **out) {
  if (!out || bytes == 0) return LBM_ERR_ARG;
  *out = nullptr;
  return cudaMallocHost(out, bytes) == cudaSuccess ? LBM_OK : LBM_ERR_OOM;
}

int lbm_host_free(void *p) {
  if (!p) return LBM_OK;
  return cudaFreeHost(p) == cudaSuccess ? LBM_OK : LBM_ERR_CUDA;
}

int lbm_pack_volume_async(lbm_sim *h, uint8_t *host_out) {
  if (!h || !host_out) return fail(h, LBM_ERR_ARG, "null");
  EntryGuard g(h);
  uint8_t *buf = nullptr;
  int slot = 0;
  int rc = next_frame(h, &buf, &slot);
  if (rc) return rc;
  h->ops->pack(h, buf);
  CKL("packVolume");
  return issue_frame_copy(h, slot, host_out);
}

int lbm_pack_volume(lbm_sim *h, uint8_t *host_out) {
  if (!h || !host_out) return fail(h, LBM_ERR_ARG, "null");
  EntryGuard g(h);
  int rc = ensure_staging(h, (size_t)h->n * 2);
  if (rc) return rc;
  h->ops->pack(h, (uint8_t *)h->staging);
  CKL("packVolume");
  CK(copy_async(h, host_out, h->staging, (size_t)h->n * 2, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return LBM_OK;
}

int lbm_render(lbm_sim *h, const lbm_sphere *sphere, const lbm_camera *cam, int width, int height,
               uint8_t *host_out) {
  if (!h || !cam || !host_out || width < 1 || height < 1 || (long long)width * height > (1LL << 28))
    return fail(h, LBM_ERR_ARG, "bad render arguments");
  EntryGuard g(h);
  int rc = ensure_staging(h, (size_t)h->n * 2);
  if (rc) return rc;
  const size_t bytes = (size_t)width * height * 4;
  if (bytes > h->imageBytes) {
    if (h->image) {
      cudaFreeAsync(h->image, h->stream);
      h->deviceBytes -= h->imageBytes;
      h->image = nullptr;
      h->imageBytes = 0;
    }
    DALLOC(h->image, bytes);
    h->imageBytes = bytes;
  }
  h->ops->pack(h, (uint8_t *)h->staging);
  CKL("packVolume");
  RenderSetup r;
  render_frame_setup(h->nx, h->ny, h->nz, sphere, cam, width, height, &r);
  CK(render_launch((const uint8_t *)h->staging, h->nx, h->ny, h->nz, r, width, height, (uint8_t *)h->image,
                   h->stream));
  h->launches++;
  CK(copy_async(h, host_out, h->image, bytes, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return LBM_OK;
}

int lbm_run_coupled(lbm_sim *h, lbm_sphere *sp, int ns, int nsteps, int frame_every, uint8_t *frames) {
  if (!h || nsteps < 0) return LBM_ERR_ARG;
  EntryGuard g(h);
  CoupledCtx c;
  int rc = coupled_prepare(h, sp, ns, frame_every > 0 && frames, c);
  if (rc) return rc;
  long long frame = 0;
  for (int s = 0; s < nsteps; s++) {
    const bool frameStep = frame_every > 0 && frames && (s + 1) % frame_every == 0;
    if ((rc = coupled_pre(h, c))) return rc;
    // a frame step's fused kernel also writes the step's RG8 volume
    h->fusePack = frameStep ? (uint8_t *)h->staging : nullptr;
    launch_fused(h);
    h->fusePack = nullptr;
    if ((rc = coupled_post(h, c))) return rc;
    h->cur = 1 - h->cur;
    if (frameStep) {
      if ((rc = coupled_frame(h, frames + frame * 2 * h->n, true))) return rc;
      frame++;
    }
  }
  if ((rc = coupled_finish(h, sp, ns))) return rc;
  return watch_after(h, nsteps);
}

int lbm_sphere_step_host(lbm_sphere *spheres, int n, double dt, double gravity, int nx, int ny, int nz) {
  if (n < 0 || (n > 0 && !spheres) || nx < 3 || ny < 3 || nz < 3) return LBM_ERR_ARG;
  for (int b = 0; b < n; b++) lbm::sphere_step_fp64(spheres[b], dt, gravity, nx, ny, nz);
  return LBM_OK;
}

int lbm_wait_frames(lbm_sim *h) {
  if (!h) return LBM_ERR_ARG;
  EntryGuard g(h);
  int rc = flush_frame_copy(h);
  if (rc) return rc;
  if (h->copyPending) {
    CK(cudaEventSynchronize(h->evCopied));
    h->copyPending = false;
    h->framePending[0] = h->framePending[1] = false;
  }
  return LBM_OK;
}

int lbm_wait_frame_slot(lbm_sim *h) {
  if (!h) return LBM_ERR_ARG;
  EntryGuard g(h);
  int rc = flush_frame_copy(h);
  if (rc) return rc;
  const int b = h->frameNext;
  if (h->framePending[b]) {
    CK(cudaEventSynchronize(h->evFrame[b]));
    h->framePending[b] = false;
  }
  return LBM_OK;
}

int lbm_synchronize(lbm_sim *h) {
  if (!h) return LBM_ERR_ARG;
  EntryGuard g(h);
  int rc = lbm_wait_frames(h);
  if (rc) return rc;
  return sync_status(h);
}

int lbm_set_nan_watchdog(lbm_sim *h, int every) {
  if (!h) return LBM_ERR_ARG;
  if (every < 0) return fail(h, LBM_ERR_ARG, "every must be >= 0 (0 turns the watchdog off)");
  h->watchEvery = every;
  h->watchSteps = 0;
  return LBM_OK;
}

int lbm_test_sequential_fill(lbm_sim *h, int on) {
  if (!h) return LBM_ERR_ARG;
  h->sequentialFill = on != 0;
  return LBM_OK;
}

int lbm_test_withhold_stage_copy(lbm_sim *h, int on) {
  if (!h) return LBM_ERR_ARG;
  h->withholdStage = on != 0;
  return LBM_OK;
}

void *lbm_stream(lbm_sim *h) { return h ? (void *)h->stream : nullptr; }

int lbm_last_sets(lbm_sim *h, int *n_fresh, int *n_dead) {
  if (!h) return LBM_ERR_ARG;
  EntryGuard g(h);
  CK(copy_async(h, h->hTotals, h->totals, 2 * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (n_fresh) *n_fresh = h->hTotals[0];
  if (n_dead) *n_dead = h->hTotals[1];
  return LBM_OK;
}

int lbm_download_sets(lbm_sim *h, int32_t *fresh, int cap_fresh, int32_t *dead, int cap_dead) {
  if (!h) return LBM_ERR_ARG;
  int nf = 0, nd = 0;
  int rc = lbm_last_sets(h, &nf, &nd);
  if (rc) return rc;
  EntryGuard g(h);
  if (fresh && cap_fresh > 0 && nf > 0)
    CK(copy_async(h, fresh, h->fresh, std::min(nf, cap_fresh) * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  if (dead && cap_dead > 0 && nd > 0)
    CK(copy_async(h, dead, h->dead, std::min(nd, cap_dead) * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return LBM_OK;
}

int lbm_launch_count(const lbm_sim *h, int64_t *count) {
  if (!h || !count) return LBM_ERR_ARG;
  *count = h->launches;
  return LBM_OK;
}

int lbm_checked_build(void) {
#ifdef LBM_CHECKED
  return 1;
#else
  return 0;
#endif
}

int lbm_fault_record(lbm_sim *h, int64_t out[4]) {
  if (!h || !out) return LBM_ERR_ARG;
  EntryGuard g(h);
  unsigned long long r[4] = {0, 0, 0, 0};
  CK(h->ops->read_fault(h, r));
  for (int j = 0; j < 4; j++) out[j] = (int64_t)r[j];
  return LBM_OK;
}

int lbm_transfer_bytes(const lbm_sim *h, uint64_t *h2d, uint64_t *d2h) {
  if (!h) return LBM_ERR_ARG;
  if (h2d) *h2d = h->h2dBytes;
  if (d2h) *d2h = h->d2hBytes;
  return LBM_OK;
}

int lbm_fused_timing(lbm_sim *h, int enable) {
  if (!h) return LBM_ERR_ARG;
  h->timing = enable != 0;
  if (enable) h->evUsed = 0;
  return LBM_OK;
}

int lbm_fused_timing_query(lbm_sim *h, double *total_ms, int64_t *launches) {
  if (!h) return LBM_ERR_ARG;
  EntryGuard g(h);
  CK(cudaStreamSynchronize(h->stream));
  double tot = 0;
  for (size_t i = 0; i < h->evUsed; i++) {
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, h->evStart[i], h->evStop[i]));
    tot += ms;
  }
  if (total_ms) *total_ms = tot;
  if (launches) *launches = (int64_t)h->evUsed;
  return LBM_OK;
}

int lbm_set_fused_config(lbm_sim *h, int rows, int zchunk) {
  if (!h) return LBM_ERR_ARG;
  if (!h->ops->shape_ok(rows) || zchunk < 1)
    return fail(h, LBM_ERR_ARG,
                "rows must be 2, 4 or 8, 4 or 6 | LBM_FUSED_COMPACT, _ASYNC or _STAGED, or 6 | LBM_FUSED_TMA or _L2PF (FP32/FP16/BF16 storage), and zchunk >= 1");
  if (h->ops->fused_smem(rows) > 227 * 1024)
    return fail(h, LBM_ERR_ARG, "that row count needs more than 227 KB of shared memory");
  h->cfg.ty = rows;
  h->cfg.zchunk = zchunk;
  return LBM_OK;
}

int lbm_set_slab(lbm_sim *h, int zoff, int own_lo, int own_hi) {
  if (!h) return LBM_ERR_ARG;
  if (own_lo < 1 || own_hi > h->nz - 2 || own_lo > own_hi || zoff < 0)
    return fail(h, LBM_ERR_ARG, "owned planes must lie in 1 .. nz - 2 and zoff >= 0");
  if (((long long)h->nx * h->ny) % 8 != 0)
    return fail(h, LBM_ERR_ARG, "slabs need nx * ny divisible by 8 (whole population blocks per plane)");
  h->slab = true;
  h->zoff = zoff;
  h->ownLo = own_lo;
  h->ownHi = own_hi;
  h->fullRetagSteps = 2;
  return LBM_OK;
}

int lbm_slab_copy_planes(lbm_sim *dst, int dst_plane, const lbm_sim *src, int src_plane, int nplanes) {
  if (!dst || !src || nplanes < 0) return LBM_ERR_ARG;
  if (dst->nx != src->nx || dst->ny != src->ny || dst->storage != src->storage)
    return fail(dst, LBM_ERR_ARG, "slabs of one scene share nx, ny and the storage form");
  if (dst_plane < 0 || src_plane < 0 || dst_plane + nplanes > dst->nz || src_plane + nplanes > src->nz)
    return fail(dst, LBM_ERR_ARG, "planes out of range");
  const long long nxny = (long long)dst->nx * dst->ny;
  if (nxny % 8 != 0) return fail(dst, LBM_ERR_ARG, "slabs need nx * ny divisible by 8");
  if (nplanes == 0) return LBM_OK;
  lbm_sim *h = dst;  // errors are reported on the destination handle
  DeviceGuard g(dst->device);
  dst->deadAhead.valid = false;
  if (dst->device != src->device) {
    // NVLink peer copies; an already-enabled peer is fine
    cudaError_t pe = cudaDeviceEnablePeerAccess(src->device, 0);
    if (pe != cudaSuccess && pe != cudaErrorPeerAccessAlreadyEnabled) return cuda_fail(dst, "peer access", pe);
    cudaGetLastError();
  }
  // the source's step must be complete
  CK(cudaStreamSynchronize(src->stream));
  const size_t pb = dst->ops->pop_bytes(), mb = dst->ops->macro_bytes();
  auto copy = [&](void *d, const void *s, size_t bytes) -> cudaError_t {
    if (dst->device == src->device) return cudaMemcpyAsync(d, s, bytes, cudaMemcpyDeviceToDevice, dst->stream);
    return cudaMemcpyPeerAsync(d, dst->device, s, src->device, bytes, dst->stream);
  };
  const long long cells = nxny * nplanes;
  const long long dc = nxny * dst_plane, sc = nxny * src_plane;
  // populations: whole 8-cell blocks of the current half
  const struct { int Q; void *d; const void *s; } pops[] = {{27, dst->F[dst->cur], src->F[src->cur]},
                                                           {7, dst->H[dst->cur], src->H[src->cur]}};
  for (const auto &p : pops) {
    const size_t blk = (size_t)32 * ((p.Q + 3) / 4) * pb;  // bytes of one 8-cell block
    CK(copy((char *)p.d + (size_t)(dc / 8) * blk, (const char *)p.s + (size_t)(sc / 8) * blk,
            (size_t)(cells / 8) * blk));
  }
  for (int a = 0; a < 5; a++)
    CK(copy((char *)dst->mac[dst->cur][a] + dc * mb, (const char *)src->mac[src->cur][a] + sc * mb,
            (size_t)cells * mb));
  CK(copy(dst->tag + dc, src->tag + sc, (size_t)cells));
  CK(cudaStreamSynchronize(dst->stream));
  dst->listsValid = false;
  return LBM_OK;
}

int lbm_get_launch_shape(const lbm_sim *h, int *shape) {
  if (!h || !shape) return LBM_ERR_ARG;
  *shape = resolve_shape(h, h->cfg.ty);
  return LBM_OK;
}

int lbm_get_fused_config(const lbm_sim *h, int *rows, int *zchunk) {
  if (!h || !rows || !zchunk) return LBM_ERR_ARG;
  *rows = h->cfg.ty;
  *zchunk = h->cfg.zchunk;
  return LBM_OK;
}

}  // extern "C"

// =====================================================================================
// Batches of scenes stepped together (declarations in include/lbm_b200.h).

struct lbm_batch {
  std::vector<lbm_sim *> sims;
  int device = 0, storage = 0;
  int rows = 4, zchunk = 32;
  std::string err;
  cudaStream_t origin = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> joins;
  void *dArgs = nullptr;  // [2][n] descriptors (FusedArgs of the storage type)
  size_t argsCap = 0;
  void *dSmall = nullptr;  // [2][n] arguments of the batched sparse kernels
  size_t smallCap = 0;
  int *dTileStart = nullptr;  // [n + 1]
  int3 *dTileGrid = nullptr;  // [n]
  int tilesCap = 0;
  uint8_t *pinned = nullptr;  // one frame of every scene
  size_t pinnedCap = 0;
  long long launches = 0;            // batched fused launches executed
  cudaGraphExec_t exec = nullptr;    // captured 2-step chunk
  std::vector<long long> execKey;    // what it baked in
  std::vector<long long> execDelta;  // per-scene launches in one chunk
};

namespace {

int bfail(lbm_batch *b, int code, const std::string &m) {
  b->err = m;
  return code;
}
int bcuda(lbm_batch *b, const char *what, cudaError_t e) {
  cudaGetLastError();
  return bfail(b, e == cudaErrorMemoryAllocation ? LBM_ERR_OOM : LBM_ERR_CUDA,
               std::string(what) + ": " + cudaGetErrorString(e));
}
#define BCK(call)                                        \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return bcuda(b, #call, e_);   \
  } while (0)
// a per-scene helper failed: carry its message to the batch
#define BSIM(h, call)                                                 \
  do {                                                                \
    int rc_ = (call);                                                 \
    if (rc_ != LBM_OK) return bfail(b, rc_, std::string("scene: ") + (h)->err); \
  } while (0)

// Per-scene descriptors for both ping-pong parities and the tile table.
int batch_tables(lbm_batch *b) {
  const int n = (int)b->sims.size();
  OpsBase *ops = b->sims[0]->ops;
  const size_t ab = ops->fused_args_bytes();
  std::vector<unsigned char> args(2 * n * ab);
  std::vector<int> start(n + 1, 0);
  std::vector<int3> grid(n);
  for (int s = 0; s < n; s++) {
    lbm_sim *h = b->sims[s];
    for (int p = 0; p < 2; p++) ops->fused_args(h, h->cur ^ p, b->zchunk, &args[(p * n + s) * ab]);
    const int rows = shape_rows(b->rows);
    grid[s] = make_int3((h->nx + 31) / 32, (h->ny + rows - 1) / rows,
                        (h->nz - 2 + b->zchunk - 1) / b->zchunk);
    long long t = (long long)start[s] + (long long)grid[s].x * grid[s].y * grid[s].z;
    if (t > (1LL << 30)) return bfail(b, LBM_ERR_CAPACITY, "too many tiles in one batch");
    start[s + 1] = (int)t;
  }
  // stream-ordered on the batch's stream (no device-wide wait)
  cudaStream_t st = b->origin;
  if (args.size() > b->argsCap) {
    if (b->dArgs) cudaFreeAsync(b->dArgs, st);
    b->dArgs = nullptr;
    BCK(cudaMallocAsync(&b->dArgs, args.size(), st));
    b->argsCap = args.size();
  }
  if (n > b->tilesCap) {
    if (b->dTileStart) cudaFreeAsync(b->dTileStart, st);
    if (b->dTileGrid) cudaFreeAsync(b->dTileGrid, st);
    b->dTileStart = nullptr;
    b->dTileGrid = nullptr;
    BCK(cudaMallocAsync(&b->dTileStart, (n + 1) * sizeof(int), st));
    BCK(cudaMallocAsync(&b->dTileGrid, n * sizeof(int3), st));
    b->tilesCap = n;
  }
  BCK(cudaMemcpyAsync(b->dArgs, args.data(), args.size(), cudaMemcpyHostToDevice, st));
  BCK(cudaMemcpyAsync(b->dTileStart, start.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice, st));
  BCK(cudaMemcpyAsync(b->dTileGrid, grid.data(), n * sizeof(int3), cudaMemcpyHostToDevice, st));
  BCK(cudaStreamSynchronize(st));  // the host vectors go out of scope
  return LBM_OK;
}

// the batch's shape for a launch: SHAPE_WIDE when any scene needs 64-bit
// population offsets
int launch_shape(const lbm_batch *b, int rows) {
  // the TMA-staged and L2-prefetch forms need every scene's tensor maps (nx
  // a multiple of 16); otherwise the batch runs the compact form of the same
  // rows
  for (lbm_sim *h : b->sims)
    if (resolve_shape(h, rows) != rows) {
      rows = resolve_shape(h, rows);
      break;
    }
  for (lbm_sim *h : b->sims)
    if (needs_wide(h->n)) return rows | SHAPE_WIDE;
  return rows;
}

int batch_tiles(const lbm_batch *b) {
  long long t = 0;
  for (lbm_sim *h : b->sims)
    t += (long long)((h->nx + 31) / 32) * ((h->ny + shape_rows(b->rows) - 1) / shape_rows(b->rows)) *
         ((h->nz - 2 + b->zchunk - 1) / b->zchunk);
  return (int)t;
}

}  // namespace

extern "C" {

int lbm_batch_create(lbm_sim *const *sims, int n, lbm_batch **out) {
  if (!sims || n < 1 || !out) return LBM_ERR_ARG;
  *out = nullptr;
  for (int s = 0; s < n; s++) {
    if (!sims[s]) return LBM_ERR_ARG;
    if (sims[s]->device != sims[0]->device || sims[s]->storage != sims[0]->storage) return LBM_ERR_ARG;
    for (int t = 0; t < s; t++)
      if (sims[t] == sims[s]) return LBM_ERR_ARG;
  }
  lbm_batch *b = new lbm_batch();
  b->sims.assign(sims, sims + n);
  b->device = sims[0]->device;
  b->storage = sims[0]->storage;
  b->rows = sims[0]->cfg.ty;
  b->zchunk = sims[0]->cfg.zchunk;
  DeviceGuard g(b->device);
  cudaError_t e = cudaStreamCreateWithFlags(&b->origin, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
  b->joins.resize(n, nullptr);
  for (int s = 0; s < n && e == cudaSuccess; s++) e = cudaEventCreateWithFlags(&b->joins[s], cudaEventDisableTiming);
  if (e != cudaSuccess) {
    cudaGetLastError();
    lbm_batch_destroy(b);
    return LBM_ERR_CUDA;
  }
  *out = b;
  return LBM_OK;
}

int lbm_batch_destroy(lbm_batch *b) {
  if (!b) return LBM_ERR_ARG;
  DeviceGuard g(b->device);
  if (b->origin) cudaStreamSynchronize(b->origin);
  if (b->dArgs) cudaFreeAsync(b->dArgs, b->origin);
  if (b->dSmall) cudaFreeAsync(b->dSmall, b->origin);
  if (b->dTileStart) cudaFreeAsync(b->dTileStart, b->origin);
  if (b->dTileGrid) cudaFreeAsync(b->dTileGrid, b->origin);
  if (b->origin) cudaStreamSynchronize(b->origin);
  for (cudaEvent_t ev : b->joins)
    if (ev) cudaEventDestroy(ev);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->origin) cudaStreamDestroy(b->origin);
  if (b->pinned) cudaFreeHost(b->pinned);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  delete b;
  return LBM_OK;
}

int lbm_batch_set_scenes(lbm_batch *b, lbm_sim *const *sims, int n) {
  if (!b || !sims || n < 1) return LBM_ERR_ARG;
  for (int s = 0; s < n; s++) {
    if (!sims[s]) return bfail(b, LBM_ERR_ARG, "scene " + std::to_string(s) + " is NULL");
    if (sims[s]->device != b->device || sims[s]->storage != b->storage)
      return bfail(b, LBM_ERR_ARG, "scene " + std::to_string(s) + " is on another device or storage form");
    for (int t = 0; t < s; t++)
      if (sims[t] == sims[s]) return bfail(b, LBM_ERR_ARG, "a scene appears twice");
  }
  DeviceGuard g(b->device);
  BCK(cudaStreamSynchronize(b->origin));
  while ((int)b->joins.size() < n) {
    cudaEvent_t ev = nullptr;
    BCK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    b->joins.push_back(ev);
  }
  b->sims.assign(sims, sims + n);
  // the captured graph names the old scenes: the next run captures anew
  if (b->exec) cudaGraphExecDestroy(b->exec);
  b->exec = nullptr;
  b->execKey.clear();
  return LBM_OK;
}

const char *lbm_batch_last_error(const lbm_batch *b) { return b ? b->err.c_str() : "null batch"; }

int lbm_batch_set_config(lbm_batch *b, int rows, int zchunk) {
  if (!b) return LBM_ERR_ARG;
  if (!b->sims[0]->ops->shape_ok(rows) || zchunk < 1)
    return bfail(b, LBM_ERR_ARG,
                 "rows must be 2, 4 or 8, 4 or 6 | LBM_FUSED_COMPACT, _ASYNC or _STAGED, or 6 | LBM_FUSED_TMA or _L2PF (FP32/FP16/BF16 storage), and zchunk >= 1");
  b->rows = rows;
  b->zchunk = zchunk;
  return LBM_OK;
}

int lbm_batch_run(lbm_batch *b, lbm_sphere *const *spheres, const int *nspheres, int nsteps,
                  int frame_every, uint8_t *const *frames, int use_graph) {
  if (!b || nsteps < 0 || !nspheres) return LBM_ERR_ARG;
  const int n = (int)b->sims.size();
  for (int s = 0; s < n; s++)
    if (nspheres[s] < 0 || nspheres[s] > LBM_MAX_SPHERES || (nspheres[s] > 0 && (!spheres || !spheres[s])))
      return bfail(b, LBM_ERR_ARG, "bad sphere arguments for scene " + std::to_string(s));
  const bool wantFrames = frame_every > 0 && frames;
  if (wantFrames)
    for (int s = 0; s < n; s++)
      if (!frames[s]) return bfail(b, LBM_ERR_ARG, "frames[" + std::to_string(s) + "] is NULL");
  DeviceGuard g(b->device);
  for (lbm_sim *sim : b->sims) sim->deadAhead.valid = false;
  OpsBase *ops = b->sims[0]->ops;
  std::vector<CoupledCtx> ctx(n);
  for (int s = 0; s < n; s++)
    BSIM(b->sims[s], coupled_prepare(b->sims[s], nspheres[s] ? spheres[s] : nullptr, nspheres[s], wantFrames,
                                     ctx[s]));
  int rc = batch_tables(b);
  if (rc) return rc;
  // the sparse kernels' arguments of every scene for both parities, and the
  // batched launches' grids (sized for the largest scene's plan bounds)
  const size_t sb = ops->small_args_bytes();
  std::vector<unsigned char> small(2 * (size_t)n * sb);
  unsigned retagCtas = 1, compactCtas = 1;
  int redX = 1, nsMax = 0;
  for (int s = 0; s < n; s++) {
    lbm_sim *h = b->sims[s];
    for (int p = 0; p < 2; p++)
      ops->small_args(h, h->cur ^ p, ctx[s].ns, ctx[s].slotCells, ctx[s].maxU, ctx[s].redChunks,
                      &small[((size_t)p * n + s) * sb]);
    retagCtas = std::max(retagCtas, std::min(nblocks(std::max(1LL, ctx[s].maxU), 256), SWEEP_CTAS));
    compactCtas = std::max(compactCtas, (unsigned)std::min<long long>(std::max(1LL, ctx[s].maxChunks), SWEEP_CTAS));
    redX = std::max(redX, ctx[s].redChunks);
    nsMax = std::max(nsMax, ctx[s].ns);
  }
  if (small.size() > b->smallCap) {
    if (b->dSmall) cudaFreeAsync(b->dSmall, b->origin);
    b->dSmall = nullptr;
    BCK(cudaMallocAsync(&b->dSmall, small.size(), b->origin));
    b->smallCap = small.size();
  }
  BCK(cudaMemcpyAsync(b->dSmall, small.data(), small.size(), cudaMemcpyHostToDevice, b->origin));
  BCK(cudaStreamSynchronize(b->origin));  // the host vector goes out of scope
  const int tiles = batch_tiles(b);
  const int ctas = std::min(tiles, ops->fused_batch_ctas(launch_shape(b, b->rows), b->device));
  const size_t ab = ops->fused_args_bytes();

  // Graph mode replays a captured chunk of 2 steps (the ping-pong halves
  // return to their parity); frames are taken between chunks, so graph mode
  // needs an even frame_every (an odd one runs eagerly).
  const bool graph = use_graph && nsteps >= 2 && (!wantFrames || frame_every % 2 == 0);
  std::vector<size_t> slot(n + 1, 0);  // pinned offset of each scene's frame
  for (int s = 0; s < n; s++) slot[s + 1] = slot[s] + (wantFrames ? 2 * (size_t)b->sims[s]->n : 0);
  if (slot[n] > b->pinnedCap) {
    // grown with headroom: page-locking is slow and a server's batch grows often
    const size_t cap = std::max(slot[n], b->pinnedCap + b->pinnedCap / 2);
    if (b->pinned) cudaFreeHost(b->pinned);
    b->pinned = nullptr;
    BCK(cudaMallocHost((void **)&b->pinned, cap));
    b->pinnedCap = cap;
  }

  // one coupled step of every scene: each kind of sparse kernel once for all
  // scenes, around the shared fused launch, all on the batch's stream
  auto emit_step = [&](int parity) -> int {
    const void *A = (const unsigned char *)b->dSmall + (size_t)parity * n * sb;
    ops->batch_pre(A, n, retagCtas, compactCtas, b->origin);
    BCK(cudaGetLastError());
    ops->fused_batch((const unsigned char *)b->dArgs + (size_t)parity * n * ab, b->dTileStart, b->dTileGrid,
                     n, launch_shape(b, b->rows), ctas, b->origin);
    BCK(cudaGetLastError());
    ops->batch_post(A, n, redX, nsMax, b->origin);
    BCK(cudaGetLastError());
    for (int s = 0; s < n; s++) b->sims[s]->cur ^= 1;
    return LBM_OK;
  };
  // RG8 volume of every scene into frames[s][idx]
  auto take_frame = [&](long long idx) -> int {
    BCK(cudaEventRecord(b->fork, b->origin));
    for (int s = 0; s < n; s++) {
      lbm_sim *h = b->sims[s];
      BCK(cudaStreamWaitEvent(h->stream, b->fork, 0));
      BSIM(h, coupled_frame(h, b->pinned + slot[s]));
      BCK(cudaEventRecord(b->joins[s], h->stream));
      BCK(cudaStreamWaitEvent(b->origin, b->joins[s], 0));
    }
    BCK(cudaStreamSynchronize(b->origin));
    for (int s = 0; s < n; s++) {
      const size_t one = 2 * (size_t)b->sims[s]->n;
      memcpy(frames[s] + (size_t)idx * one, b->pinned + slot[s], one);
    }
    return LBM_OK;
  };

  // the captured 2-step graph, reused while nothing it baked in has changed
  if (graph) {
    std::vector<long long> key = {b->rows, b->zchunk, (long long)(uintptr_t)b->dArgs,
                                  (long long)(uintptr_t)b->dTileStart, ctas, (long long)(uintptr_t)b->dSmall,
                                  retagCtas, compactCtas, redX, nsMax};
    for (int s = 0; s < n; s++) {
      lbm_sim *h = b->sims[s];
      const long long v[] = {(long long)(uintptr_t)h,           h->cur,      ctx[s].ns,
                             ctx[s].slotCells,                  ctx[s].maxU, ctx[s].maxChunks,
                             ctx[s].redChunks,                  (long long)(uintptr_t)h->impAcc,
                             (long long)(uintptr_t)h->partials, (long long)(uintptr_t)h->counts};
      key.insert(key.end(), v, v + 10);
    }
    if (!b->exec || key != b->execKey) {
      if (b->exec) cudaGraphExecDestroy(b->exec);
      b->exec = nullptr;
      std::vector<long long> l0(n);
      for (int s = 0; s < n; s++) l0[s] = b->sims[s]->launches;
      cudaGraph_t gr = nullptr;
      BCK(cudaStreamBeginCapture(b->origin, cudaStreamCaptureModeThreadLocal));
      int erc = emit_step(0);
      if (erc == LBM_OK) erc = emit_step(1);
      cudaError_t ce = cudaStreamEndCapture(b->origin, &gr);
      b->execDelta.assign(n, 0);
      for (int s = 0; s < n; s++) {
        b->execDelta[s] = b->sims[s]->launches - l0[s];
        b->sims[s]->launches = l0[s];  // counted when the graph runs
      }
      if (erc != LBM_OK || ce != cudaSuccess) {
        if (gr) cudaGraphDestroy(gr);
        cudaGetLastError();
        if (erc != LBM_OK) return erc;
        return bcuda(b, "cudaStreamEndCapture", ce);
      }
      ce = cudaGraphInstantiate(&b->exec, gr, 0);
      cudaGraphDestroy(gr);
      if (ce != cudaSuccess) {
        b->exec = nullptr;
        return bcuda(b, "cudaGraphInstantiate", ce);
      }
      b->execKey = key;
    }
  }

  long long done = 0;
  while (done < nsteps) {
    if (graph && nsteps - done >= 2) {
      BCK(cudaGraphLaunch(b->exec, b->origin));
      for (int s = 0; s < n; s++) b->sims[s]->launches += b->execDelta[s];
      b->launches += 2;
      done += 2;
    } else {
      if ((rc = emit_step((int)(done & 1)))) return rc;
      b->launches++;
      done++;
    }
    if (wantFrames && done % frame_every == 0 && (rc = take_frame(done / frame_every - 1))) return rc;
  }
  BCK(cudaStreamSynchronize(b->origin));
  for (int s = 0; s < n; s++)
    BSIM(b->sims[s], coupled_finish(b->sims[s], nspheres[s] ? spheres[s] : nullptr, nspheres[s]));
  // every scene's watchdog advances and scans; the first scene that reports
  // gives the batch's status and message
  int first = LBM_OK;
  std::string firstMsg;
  for (int s = 0; s < n; s++) {
    const int rc_ = watch_after(b->sims[s], nsteps);
    if (rc_ != LBM_OK && first == LBM_OK) {
      first = rc_;
      firstMsg = "scene " + std::to_string(s) + ": " + b->sims[s]->err;
    }
  }
  if (first != LBM_OK) return bfail(b, first, firstMsg);
  return LBM_OK;
}

int lbm_batch_time_fused(lbm_batch *b, int rows, int zchunk, int reps, double *ms) {
  if (!b || !ms || reps < 1) return LBM_ERR_ARG;
  if (!b->sims[0]->ops->shape_ok(rows) || zchunk < 1)
    return bfail(b, LBM_ERR_ARG,
                 "rows must be 2, 4 or 8, 4 or 6 | LBM_FUSED_COMPACT, _ASYNC or _STAGED, or 6 | LBM_FUSED_TMA or _L2PF (FP32/FP16/BF16 storage), and zchunk >= 1");
  DeviceGuard g(b->device);
  const int keepRows = b->rows, keepZ = b->zchunk;
  b->rows = rows;
  b->zchunk = zchunk;
  int rc = batch_tables(b);
  OpsBase *ops = b->sims[0]->ops;
  const int ctas = std::min(batch_tiles(b), ops->fused_batch_ctas(launch_shape(b, rows), b->device));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (rc == LBM_OK) {
    for (lbm_sim *h : b->sims) cudaStreamSynchronize(h->stream);
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    ops->fused_batch(b->dArgs, b->dTileStart, b->dTileGrid, (int)b->sims.size(), launch_shape(b, rows), ctas,
                     b->origin);
    cudaEventRecord(e0, b->origin);
    for (int r = 0; r < reps; r++)
      ops->fused_batch(b->dArgs, b->dTileStart, b->dTileGrid, (int)b->sims.size(), launch_shape(b, rows), ctas,
                     b->origin);
    cudaEventRecord(e1, b->origin);
    cudaError_t e = cudaEventSynchronize(e1);
    float t = 0;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
    if (e != cudaSuccess) rc = bcuda(b, "timing the batched fused kernel", e);
    *ms = (double)t / reps;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  b->rows = keepRows;
  b->zchunk = keepZ;
  return rc;
}

int lbm_batch_launch_count(const lbm_batch *b, int64_t *count) {
  if (!b || !count) return LBM_ERR_ARG;
  *count = b->launches;
  return LBM_OK;
}

}  // extern "C"
