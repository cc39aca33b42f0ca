// Device-side voxelisation of a rigid triangle mesh: the cells a closed mesh
// contains and their surface velocity, for the generic-solid path (the
// reference's solid interface is mesh-agnostic, README.md:65-73; the sphere's
// surfaceVelocity, src/solid.js:57-66, is the rigid-body formula used here).
//
// A cell is inside when the ray from its centre (x + 0.5, y + 0.5, z + 0.5)
// towards +x crosses the mesh an odd number of times.  A triangle is crossed
// when the ray's (y, z) lies in the triangle's projection on the yz plane --
// edge functions in FP64 with a top-left rule for points on an edge, so a
// ray through an edge shared by two triangles counts once -- and the plane's
// x at that (y, z) lies beyond the centre.  Every operation is rounded
// explicitly (no contraction), so a host restatement in double arithmetic
// decides every cell the same way.
#pragma once

#include "lbm_core.cuh"

namespace lbm {

struct MeshMotion {
  double cx, cy, cz;  // the point the angular velocity turns about
  double vx, vy, vz;  // linear velocity
  double wx, wy, wz;  // angular velocity
};

constexpr int MESH_TILE = 128;  // triangles staged in shared memory at a time
constexpr int MESH_THREADS = 256;

__device__ __forceinline__ double m_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double m_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double m_add(double a, double b) { return __dadd_rn(a, b); }

// edge function of the edge P -> Q at S in the yz plane
__device__ __forceinline__ double m_edge(double py, double pz, double qy, double qz, double sy, double sz) {
  return m_sub(m_mul(m_sub(qy, py), m_sub(sz, pz)), m_mul(m_sub(qz, pz), m_sub(sy, py)));
}
// top-left rule for a counter-clockwise triangle (y horizontal, z vertical):
// an edge whose interior side holds the points exactly on it
__device__ __forceinline__ bool m_top_left(double py, double pz, double qy, double qz) {
  const double dy = m_sub(qy, py), dz = m_sub(qz, pz);
  return (dz == 0.0 && dy < 0.0) || dz < 0.0;
}

// does the +x ray from (px, py, pz) cross triangle t (9 doubles: A, B, C)?
__device__ __forceinline__ bool ray_crosses(const double *t, double px, double py, double pz) {
  const double ax = t[0], ay = t[1], az = t[2], bx = t[3], by = t[4], bz = t[5], cx = t[6], cy = t[7], cz = t[8];
  // plane normal (B - A) x (C - A); its x part is twice the projected area
  const double nx = m_sub(m_mul(m_sub(by, ay), m_sub(cz, az)), m_mul(m_sub(bz, az), m_sub(cy, ay)));
  if (nx == 0.0) return false;  // edge-on to the ray
  // the projection counter-clockwise: B and C exchanged when it is not
  double y1 = by, z1 = bz, y2 = cy, z2 = cz;
  if (nx < 0.0) {
    y1 = cy;
    z1 = cz;
    y2 = by;
    z2 = bz;
  }
  const double e0 = m_edge(ay, az, y1, z1, py, pz);
  const double e1 = m_edge(y1, z1, y2, z2, py, pz);
  const double e2 = m_edge(y2, z2, ay, az, py, pz);
  const bool in0 = e0 > 0.0 || (e0 == 0.0 && m_top_left(ay, az, y1, z1));
  const bool in1 = e1 > 0.0 || (e1 == 0.0 && m_top_left(y1, z1, y2, z2));
  const bool in2 = e2 > 0.0 || (e2 == 0.0 && m_top_left(y2, z2, ay, az));
  if (!(in0 && in1 && in2)) return false;
  const double ny = m_sub(m_mul(m_sub(bz, az), m_sub(cx, ax)), m_mul(m_sub(bx, ax), m_sub(cz, az)));
  const double nz = m_sub(m_mul(m_sub(bx, ax), m_sub(cy, ay)), m_mul(m_sub(by, ay), m_sub(cx, ax)));
  const double xh = m_sub(ax, __ddiv_rn(m_add(m_mul(ny, m_sub(py, ay)), m_mul(nz, m_sub(pz, az))), nx));
  return xh > px;
}

// mask and surface velocity of the cells of box [lo, lo + dim) (the rest of
// the grid is cleared beforehand); one thread per cell, triangles staged in
// shared memory tile by tile
static __global__ void __launch_bounds__(MESH_THREADS)
    k_voxelize_mesh(const double *__restrict__ tri, int ntri, int nx, int ny, int3 lo, int3 dim, MeshMotion m,
                    uint8_t *mask, float *us) {
  __shared__ double st[MESH_TILE * 9];
  const long long cells = (long long)dim.x * dim.y * dim.z;
  const long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const bool active = l < cells;
  int x = 0, y = 0, z = 0;
  if (active) {
    x = lo.x + (int)(l % dim.x);
    y = lo.y + (int)((l / dim.x) % dim.y);
    z = lo.z + (int)(l / ((long long)dim.x * dim.y));
  }
  const double px = (double)x + 0.5, py = (double)y + 0.5, pz = (double)z + 0.5;
  int crossings = 0;
  for (int t0 = 0; t0 < ntri; t0 += MESH_TILE) {
    const int nt = min(MESH_TILE, ntri - t0);
    __syncthreads();
    for (int j = threadIdx.x; j < nt * 9; j += blockDim.x) st[j] = tri[(long long)t0 * 9 + j];
    __syncthreads();
    if (active)
      for (int t = 0; t < nt; t++) crossings += ray_crosses(st + 9 * t, px, py, pz) ? 1 : 0;
  }
  if (!active) return;
  const long long i = ((long long)z * ny + y) * nx + x;
  const bool inside = crossings & 1;
  mask[i] = inside ? 1 : 0;
  if (inside && us) {
    // u_body + omega x r, as RigidSphere.surfaceVelocity (src/solid.js:57-66)
    const double rx = m_sub(px, m.cx), ry = m_sub(py, m.cy), rz = m_sub(pz, m.cz);
    us[3 * i + 0] = (float)m_add(m.vx, m_sub(m_mul(m.wy, rz), m_mul(m.wz, ry)));
    us[3 * i + 1] = (float)m_add(m.vy, m_sub(m_mul(m.wz, rx), m_mul(m.wx, rz)));
    us[3 * i + 2] = (float)m_add(m.vz, m_sub(m_mul(m.wx, ry), m_mul(m.wy, rx)));
  }
}

}  // namespace lbm
