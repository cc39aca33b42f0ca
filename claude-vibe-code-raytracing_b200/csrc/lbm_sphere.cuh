// RigidSphere.step (src/solid.js:104-210) in FP64, shared by the device and
// the host side of the library.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

#include <cmath>

#include "lbm_b200.h"

namespace lbm {

// RigidSphere.step(dt, gravity) (src/solid.js:104-210) in FP64, in the
// reference's evaluation order: one rounding per operation (round-to-nearest
// intrinsics on the device; the host side of the library is compiled without
// FMA contraction).  Shared by the device-resident loop (k_sphere_step) and
// the host entry point lbm_sphere_step_host.
struct F64 {
  __host__ __device__ static double add(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
  }
  __host__ __device__ static double sub(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
  }
  __host__ __device__ static double mul(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
  }
  __host__ __device__ static double div(double a, double b) {
#ifdef __CUDA_ARCH__
    return __ddiv_rn(a, b);
#else
    return a / b;
#endif
  }
  __host__ __device__ static double sqrt_(double a) {
#ifdef __CUDA_ARCH__
    return __dsqrt_rn(a);
#else
    return std::sqrt(a);
#endif
  }
};
// Math.max(0, v) / Math.min(0, v): NaN propagates, +0 beats -0 (max) and -0
// beats +0 (min)
__host__ __device__ inline double js_max0(double v) {
  if (v != v) return v;
  if (v == 0) return signbit(v) ? 0.0 : v;
  return v > 0 ? v : 0.0;
}
__host__ __device__ inline double js_min0(double v) {
  if (v != v) return v;
  if (v == 0) return signbit(v) ? v : 0.0;
  return v < 0 ? v : 0.0;
}

__host__ __device__ inline void sphere_step_fp64(lbm_sphere &s, double dt, double gravity, int nx, int ny, int nz) {
  using M = F64;
  s.Fy = M::add(s.Fy, M::mul(s.mass, gravity));
  if (s.dragging) {
    double k = M::mul(0.004, s.mass);
    double cD = M::mul(2.0, M::sqrt_(M::mul(k, s.mass)));
    s.Fx = M::add(s.Fx, M::sub(M::mul(k, M::sub(s.dragTargetX, s.cx)), M::mul(cD, s.vx)));
    s.Fy = M::add(s.Fy, M::sub(M::mul(k, M::sub(s.dragTargetY, s.cy)), M::mul(cD, s.vy)));
    s.Fz = M::add(s.Fz, M::sub(M::mul(k, M::sub(s.dragTargetZ, s.cz)), M::mul(cD, s.vz)));
  }
  // `gravity || 0.001`: zero and NaN select the fallback
  double gsel = (gravity == 0 || gravity != gravity) ? 0.001 : gravity;
  double accCap = M::mul(3.5, fabs(gsel));
  {
    double ax = M::div(s.Fx, s.mass);
    double ay = M::div(s.Fy, s.mass);
    double az = M::div(s.Fz, s.mass);
    double a2 = M::add(M::add(M::mul(ax, ax), M::mul(ay, ay)), M::mul(az, az));
    double c2 = M::mul(accCap, accCap);
    double sc = a2 > c2 ? M::div(accCap, M::sqrt_(a2)) : 1.0;
    s.vx = M::add(s.vx, M::mul(M::mul(dt, ax), sc));
    s.vy = M::add(s.vy, M::mul(M::mul(dt, ay), sc));
    s.vz = M::add(s.vz, M::mul(M::mul(dt, az), sc));
  }
  s.wx = M::add(s.wx, M::div(M::mul(dt, s.Tx), s.I));
  s.wy = M::add(s.wy, M::div(M::mul(dt, s.Ty), s.I));
  s.wz = M::add(s.wz, M::div(M::mul(dt, s.Tz), s.I));
  const double BODY_UMAX = 0.08;
  double sp2 = M::add(M::add(M::mul(s.vx, s.vx), M::mul(s.vy, s.vy)), M::mul(s.vz, s.vz));
  if (sp2 > M::mul(BODY_UMAX, BODY_UMAX)) {
    double sc = M::div(BODY_UMAX, M::sqrt_(sp2));
    s.vx = M::mul(s.vx, sc);
    s.vy = M::mul(s.vy, sc);
    s.vz = M::mul(s.vz, sc);
  }
  s.vx = M::mul(s.vx, 0.98);
  s.vy = M::mul(s.vy, 0.98);
  s.vz = M::mul(s.vz, 0.98);
  s.wx = M::mul(s.wx, 0.95);
  s.wy = M::mul(s.wy, 0.95);
  s.wz = M::mul(s.wz, 0.95);
  const double SNAP = 0.0001;
  if (fabs(s.vx) < SNAP) s.vx = 0;
  if (fabs(s.vy) < SNAP) s.vy = 0;
  if (fabs(s.vz) < SNAP) s.vz = 0;
  if (fabs(s.wx) < SNAP) s.wx = 0;
  if (fabs(s.wy) < SNAP) s.wy = 0;
  if (fabs(s.wz) < SNAP) s.wz = 0;
  s.cx = M::add(s.cx, M::mul(dt, s.vx));
  s.cy = M::add(s.cy, M::mul(dt, s.vy));
  s.cz = M::add(s.cz, M::mul(dt, s.vz));
  double m = M::add(s.r, 1.5);
  double limX = M::sub((double)(nx - 1), m), limY = M::sub((double)(ny - 1), m);
  double limZ = M::sub((double)(nz - 1), m);
  if (s.cx < m) { s.cx = m; s.vx = js_max0(s.vx); }
  if (s.cx > limX) { s.cx = limX; s.vx = js_min0(s.vx); }
  if (s.cy < m) { s.cy = m; s.vy = js_max0(s.vy); }
  if (s.cy > limY) { s.cy = limY; s.vy = js_min0(s.vy); }
  if (s.cz < m) { s.cz = m; s.vz = js_max0(s.vz); }
  if (s.cz > limZ) { s.cz = limZ; s.vz = js_min0(s.vz); }
  s.Fx = s.Fy = s.Fz = 0;
  s.Tx = s.Ty = s.Tz = 0;
}

}  // namespace lbm
