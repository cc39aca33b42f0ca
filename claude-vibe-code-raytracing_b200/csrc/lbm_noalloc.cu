// Allocation-free variant of the dead-cell sweep (lbm_absorb_dead_cells_noalloc,
// declared in include/lbm_b200.h).
//
// Some callers cannot allocate device memory at the point where they need the
// sweep: an engine that hands out all device memory from its own fixed pool and
// forbids allocation elsewhere, a host process whose allocator is owned by
// another runtime, or a loop that must not pay the device-wide synchronisation a
// cudaMalloc / cudaFree can cost.  This entry point works on device arrays the
// caller already owns and keeps its own scratch -- the per-chunk counts, the
// totals and the scan-ordered cell lists of the compaction -- in one fixed,
// file-scope device array.  It calls no allocator, host or device.
//
// Limit: the search box (the union of the spheres' bounding boxes, clamped to
// the interior) may hold at most NOALLOC_MAX_BOX = 2^20 cells, e.g. one sphere
// of radius up to ~49 cells.  Every GPU that loads the library holds the array
// (about 8.4 MB) until the process exits.
//
// Set-up: the first call on each device, with that device current, looks up
// the array's device address (cudaGetSymbolAddress, which also loads this
// module onto the device).  Make that first call before any stream capture.
//
// Sharing: all calls on a device use the same array, which keeps the last
// call's contents.  Everything a call reads there it has written first (the
// plan, the counts of the chunks in use, the totals and the list entries below
// the totals), so nothing needs clearing between calls.  Calls whose kernels
// overlap on the GPU (different streams, or several host threads) race on the
// array and must be serialised by the caller.
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <mutex>

#include "lbm_kernels.cuh"
#include "lbm_state.h"

using namespace lbm;

namespace {

constexpr long long NOALLOC_MAX_BOX = 1LL << 20;  // cells of the search box
constexpr int NOALLOC_MAX_CHUNKS = (int)(NOALLOC_MAX_BOX / COMPACT_CHUNK);
constexpr int NOALLOC_MAX_DEVICES = 64;

struct NoAllocScratch {
  Plan plan;
  int totals[2];
  int2 counts[NOALLOC_MAX_CHUNKS];
  int fresh[NOALLOC_MAX_BOX];
  int dead[NOALLOC_MAX_BOX];
};

std::mutex g_mu;
NoAllocScratch *g_scratch[NOALLOC_MAX_DEVICES] = {nullptr};

int fail(char *err, size_t errlen, int code, const char *fmt, ...) {
  if (err && errlen > 0) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, errlen, fmt, ap);
    va_end(ap);
  }
  return code;
}

__global__ void k_noalloc_set_plan(Plan *dst, const __grid_constant__ Plan src) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *dst = src;
}

bool on_device(const void *p) {
  cudaPointerAttributes at;
  if (!p || cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

}  // namespace

// The scratch.  In host code this name only identifies the array for
// cudaGetSymbolAddress; it is not a device address.
static __device__ __align__(256) unsigned char lbm_noalloc_scratch[sizeof(NoAllocScratch)];

extern "C" int lbm_absorb_dead_cells_noalloc(int nx, int ny, int nz, double rhoL, double rhoG,
                                             const uint8_t *tag, const uint8_t *tagPrev,
                                             const float *phi, const float *ux, const float *uy,
                                             const float *uz, const lbm_sphere *spheres,
                                             int nspheres, double *out, void *stream, char *err,
                                             size_t errlen) {
  if (err && errlen > 0) err[0] = '\0';
  if (nx < 3 || ny < 3 || nz < 3 || (long long)nx * ny * nz >= (1LL << 31))
    return fail(err, errlen, LBM_ERR_ARG, "grid %d x %d x %d out of range", nx, ny, nz);
  if (nspheres < 0 || nspheres > LBM_MAX_SPHERES)
    return fail(err, errlen, LBM_ERR_ARG, "nspheres %d outside [0, %d]", nspheres, LBM_MAX_SPHERES);
  if (nspheres == 0) return LBM_OK;
  if (!spheres) return fail(err, errlen, LBM_ERR_ARG, "spheres is NULL");

  // search box: dead cells are SOLID, so they lie inside the spheres' boxes
  Plan P;
  memset(&P, 0, sizeof(P));
  Box U{{1, 1, 1}, {0, 0, 0}};
  P.ss.nsph = nspheres;
  for (int b = 0; b < nspheres; b++) {
    SphereDesc &d = P.ss.sph[b];
    d.cx = spheres[b].cx;
    d.cy = spheres[b].cy;
    d.cz = spheres[b].cz;
    d.r = spheres[b].r;
    d.vx = spheres[b].vx;
    d.vy = spheres[b].vy;
    d.vz = spheres[b].vz;
    d.wx = spheres[b].wx;
    d.wy = spheres[b].wy;
    d.wz = spheres[b].wz;
    U = box_union(U, sphere_box(d.cx, d.cy, d.cz, d.r, nx, ny, nz));
  }
  const long long cells = box_cells(U);
  if (cells > NOALLOC_MAX_BOX)
    return fail(err, errlen, LBM_ERR_CAPACITY,
                "the spheres' search box holds %lld cells; this entry point handles at most %lld "
                "(use lbm_absorb_dead_cells for larger spheres)",
                cells, NOALLOC_MAX_BOX);
  if (cells == 0) {
    // no interior cell can be SOLID: the impulse is zero
    if (!on_device(out)) return fail(err, errlen, LBM_ERR_ARG, "out must be a device pointer");
    cudaError_t e = cudaMemsetAsync(out, 0, (size_t)nspheres * 6 * sizeof(double), (cudaStream_t)stream);
    if (e != cudaSuccess) return fail(err, errlen, LBM_ERR_CUDA, "cudaMemsetAsync: %s", cudaGetErrorString(e));
    return LBM_OK;
  }
  const void *dptrs[] = {tag, tagPrev, phi, ux, uy, uz, out};
  for (const void *p : dptrs)
    if (!on_device(p))
      return fail(err, errlen, LBM_ERR_ARG, "tag, tagPrev, phi, ux, uy, uz and out must be device pointers");
  P.U = U;
  P.ucells = cells;
  P.nchunks = (int)((cells + COMPACT_CHUNK - 1) / COMPACT_CHUNK);

  // set-up, once per device, with that device current
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES)
    return fail(err, errlen, LBM_ERR_CUDA, "no usable current CUDA device");
  NoAllocScratch *S = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch[dev]) {
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, lbm_noalloc_scratch);
      if (e != cudaSuccess || !p) {
        cudaGetLastError();
        return fail(err, errlen, LBM_ERR_CUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
      }
      g_scratch[dev] = (NoAllocScratch *)p;
    }
    S = g_scratch[dev];
  }

  cudaStream_t s = (cudaStream_t)stream;
  const unsigned grid = (unsigned)P.nchunks;  // 1 .. NOALLOC_MAX_CHUNKS
  k_noalloc_set_plan<<<1, 1, 0, s>>>(&S->plan, P);
  k_compact_count<<<grid, COMPACT_THREADS, 0, s>>>(tag, tagPrev, nx, ny, &S->plan, S->counts);
  k_compact_scan<<<1, 1024, 0, s>>>(S->counts, &S->plan, S->totals);
  k_compact_emit<<<grid, COMPACT_THREADS, 0, s>>>(tag, tagPrev, nx, ny, &S->plan, S->counts, S->fresh,
                                                   S->dead, (int)NOALLOC_MAX_BOX);
  k_absorb_dead<float><<<nspheres, DEAD_THREADS, 0, s>>>(phi, ux, uy, uz, nx, ny, S->dead, S->totals,
                                                          (int)NOALLOC_MAX_BOX, rhoL, rhoG,
                                                          &S->plan.ss, out);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(err, errlen, LBM_ERR_CUDA, "launch: %s", cudaGetErrorString(e));
  return LBM_OK;
}
