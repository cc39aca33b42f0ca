// Headless raymarcher of the RG8 volume (lbm_render_volume / lbm_render in
// include/lbm_b200.h).
//
// The reference draws each frame with a WebGL2 fragment shader over a
// fullscreen quad (src/render.js:19-268), reading the packed volume
// (Sim.packVolume, src/sim.js:586-600) as an RG8 3D texture with linear
// filtering and clamp-to-edge (src/render.js:391-399), from an orbit camera
// (src/render.js:405-448, 484-513).  Here one CUDA thread per pixel evaluates
// the same shading in FP32: the ray from the inverse view-projection, the
// tank (AABB) and sphere intersections, the 48-step march for the phi = 0.5
// crossing with the per-pixel jitter, the gradient normal, Fresnel-mixed
// reflection and refraction with Beer-Lambert tinting, the sky and sphere
// shading, tonemap and gamma; the colour is written as RGBA8 (top row first)
// into a device buffer instead of a canvas.  Texture filtering is done in
// software with full-precision weights (texel centres at (i + 0.5) / n).
//
// This file is compiled without FMA contraction (-fmad=false) so its
// arithmetic follows the shader's operation order; see csrc/Makefile.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <cuda_runtime.h>

#include "lbm_b200.h"
#include "lbm_render.h"

namespace lbm {

namespace {

struct V3 {
  float x, y, z;
};
__device__ __forceinline__ V3 v3(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ V3 operator/(V3 a, V3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 normalize(V3 a) { return a * (1.0f / sqrtf(dot(a, a))); }
__device__ __forceinline__ V3 vmin(V3 a, V3 b) { return {fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)}; }
__device__ __forceinline__ V3 vmax(V3 a, V3 b) { return {fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)}; }
__device__ __forceinline__ float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }
// GLSL mix: x (1 - a) + y a
__device__ __forceinline__ V3 mix(V3 x, V3 y, float a) { return x * (1.0f - a) + y * a; }
__device__ __forceinline__ float smooth01(float t) {
  t = clampf(t, 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}
__device__ __forceinline__ V3 reflect(V3 i, V3 n) { return i - 2.0f * dot(n, i) * n; }
__device__ __forceinline__ V3 refract(V3 i, V3 n, float eta) {
  const float d = dot(n, i);
  const float k = 1.0f - eta * eta * (1.0f - d * d);
  if (k < 0.0f) return v3(0.0f, 0.0f, 0.0f);
  return eta * i - (eta * d + sqrtf(k)) * n;
}

struct Frame {
  const uint8_t *vol;
  int nx, ny, nz, width, height;
  float inv[16];  // inverse view-projection, column-major
  V3 cam, gridInv, boxMax, light, sphC;
  float sphR;
  uint8_t *out;
};

// texture(uVol, uvw).r: trilinear over the R channel, clamp to edge
__device__ float sample_phi(const Frame &f, V3 wp) {
  const V3 uvw = wp / f.boxMax;
  const float u = uvw.x * (float)f.nx - 0.5f, v = uvw.y * (float)f.ny - 0.5f, w = uvw.z * (float)f.nz - 0.5f;
  const float fu = floorf(u), fv = floorf(v), fw = floorf(w);
  const float a = u - fu, b = v - fv, c = w - fw;
  int x0 = (int)fu, y0 = (int)fv, z0 = (int)fw;
  int x1 = x0 + 1, y1 = y0 + 1, z1 = z0 + 1;
  x0 = min(max(x0, 0), f.nx - 1);
  x1 = min(max(x1, 0), f.nx - 1);
  y0 = min(max(y0, 0), f.ny - 1);
  y1 = min(max(y1, 0), f.ny - 1);
  z0 = min(max(z0, 0), f.nz - 1);
  z1 = min(max(z1, 0), f.nz - 1);
  auto t = [&](int x, int y, int z) -> float {
    return (float)__ldg(f.vol + 2 * (((long long)z * f.ny + y) * f.nx + x)) * (1.0f / 255.0f);
  };
  const float c00 = t(x0, y0, z0) * (1.0f - a) + t(x1, y0, z0) * a;
  const float c10 = t(x0, y1, z0) * (1.0f - a) + t(x1, y1, z0) * a;
  const float c01 = t(x0, y0, z1) * (1.0f - a) + t(x1, y0, z1) * a;
  const float c11 = t(x0, y1, z1) * (1.0f - a) + t(x1, y1, z1) * a;
  const float c0 = c00 * (1.0f - b) + c10 * b;
  const float c1 = c01 * (1.0f - b) + c11 * b;
  return c0 * (1.0f - c) + c1 * c;
}

__device__ V3 grad_phi(const Frame &f, V3 wp) {
  const V3 e = f.boxMax * f.gridInv;
  return v3(sample_phi(f, wp + v3(e.x, 0, 0)) - sample_phi(f, wp - v3(e.x, 0, 0)),
            sample_phi(f, wp + v3(0, e.y, 0)) - sample_phi(f, wp - v3(0, e.y, 0)),
            sample_phi(f, wp + v3(0, 0, e.z)) - sample_phi(f, wp - v3(0, 0, e.z)));
}

__device__ void intersect_aabb(V3 ro, V3 rd, V3 bmin, V3 bmax, float &tn, float &tf) {
  const V3 inv = v3(1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z);
  const V3 t1 = (bmin - ro) * inv, t2 = (bmax - ro) * inv;
  const V3 lo = vmin(t1, t2), hi = vmax(t1, t2);
  tn = fmaxf(fmaxf(lo.x, lo.y), lo.z);
  tf = fminf(fminf(hi.x, hi.y), hi.z);
}

__device__ float intersect_sphere(V3 ro, V3 rd, V3 c, float r) {
  const V3 oc = ro - c;
  const float b = dot(oc, rd);
  const float cc = dot(oc, oc) - r * r;
  float d = b * b - cc;
  if (d < 0.0f) return -1.0f;
  d = sqrtf(d);
  float t = -b - d;
  if (t < 0.0f) t = -b + d;
  return t;
}

__device__ V3 sky_color(const Frame &f, V3 rd) {
  const float t = clampf(-rd.y * 0.5f + 0.5f, 0.0f, 1.0f);
  V3 sky = mix(v3(0.72f, 0.78f, 0.86f), v3(0.18f, 0.32f, 0.55f), smooth01(t));
  const float sun = powf(fmaxf(dot(rd, -f.light), 0.0f), 96.0f);
  return sky + v3(1.0f, 0.92f, 0.72f) * (sun * 0.9f);
}

__device__ V3 shade_sphere(const Frame &f, V3 wp, V3 rd) {
  const V3 n = normalize(wp - f.sphC);
  const float lambert = fmaxf(dot(n, -f.light), 0.0f);
  V3 col = v3(0.95f, 0.78f, 0.35f) * (0.22f + 0.85f * lambert);
  const V3 h = normalize(-f.light - rd);
  col = col + v3(1.0f, 1.0f, 1.0f) * (powf(fmaxf(dot(h, n), 0.0f), 48.0f) * 0.55f);
  const float rim = powf(1.0f - fmaxf(dot(-rd, n), 0.0f), 3.0f);
  return col + v3(1.0f, 0.85f, 0.6f) * (rim * 0.18f);
}

__device__ V3 trace_backdrop(const Frame &f, V3 ro, V3 rd, float &outT) {
  float tn, tf;
  intersect_aabb(ro, rd, v3(0, 0, 0), f.boxMax, tn, tf);
  const float tExit = fmaxf(tf, 0.0f);
  const float tS = intersect_sphere(ro, rd, f.sphC, f.sphR);
  if (tS > 0.0f && tS < tExit) {
    outT = tS;
    return shade_sphere(f, ro + tS * rd, rd);
  }
  outT = tExit;
  return sky_color(f, rd);
}

__device__ V3 water_attenuate(V3 back, float d) {
  const V3 trans = v3(expf(-2.6f * d), expf(-0.55f * d), expf(-0.25f * d));
  return trans * back + (v3(1.0f, 1.0f, 1.0f) - trans) * v3(0.03f, 0.11f, 0.16f);
}

__device__ float fresnel_schlick(float cosI, float f0) { return f0 + (1.0f - f0) * powf(1.0f - cosI, 5.0f); }

__device__ __forceinline__ V3 mat_point(const float *m, float x, float y, float z) {
  float o[4];
  for (int i = 0; i < 4; i++) o[i] = m[i] * x + m[4 + i] * y + m[8 + i] * z + m[12 + i] * 1.0f;
  return v3(o[0] / o[3], o[1] / o[3], o[2] / o[3]);
}

__device__ V3 tonemap(V3 c) {
  c = c / (c + v3(1.0f, 1.0f, 1.0f));
  return v3(powf(c.x, 1.0f / 2.2f), powf(c.y, 1.0f / 2.2f), powf(c.z, 1.0f / 2.2f));
}

__global__ void k_render(const Frame f) {
  const int px = blockIdx.x * blockDim.x + threadIdx.x;
  const int py = blockIdx.y * blockDim.y + threadIdx.y;  // window row, 0 at the bottom
  if (px >= f.width || py >= f.height) return;
  const float uvx = ((float)px + 0.5f) / (float)f.width, uvy = ((float)py + 0.5f) / (float)f.height;
  const float ndx = uvx * 2.0f - 1.0f, ndy = uvy * 2.0f - 1.0f;
  const V3 wNear = mat_point(f.inv, ndx, ndy, -1.0f);
  const V3 wFar = mat_point(f.inv, ndx, ndy, 1.0f);
  const V3 rd = normalize(wFar - wNear);
  const V3 ro = f.cam;

  V3 col;
  float tn, tf;
  intersect_aabb(ro, rd, v3(0, 0, 0), f.boxMax, tn, tf);
  const float tEnter = fmaxf(tn, 0.0f), tExit = tf;
  if (tExit < tEnter) {
    col = tonemap(sky_color(f, rd));
  } else {
    const float tSphereRaw = intersect_sphere(ro, rd, f.sphC, f.sphR);
    const float tSphere = (tSphereRaw > tEnter && tSphereRaw < tExit) ? tSphereRaw : -1.0f;
    const float tEnd = tSphere > 0.0f ? tSphere : tExit;
    const float epsT = 0.002f * (tEnd - tEnter);
    float prevT = tEnter + epsT;
    float prevPhi = sample_phi(f, ro + prevT * rd);
    const bool startInWater = prevPhi > 0.5f;
    const int STEPS = 48;
    const float dt = (tEnd - prevT) / (float)STEPS;
    const float s = sinf(uvx * 12.9898f + uvy * 78.233f) * 43758.5453f;
    const float jit = s - floorf(s);
    float tSurface = -1.0f;
    for (int i = 0; i < STEPS; i++) {
      const float t = prevT + ((float)i + 0.5f + jit) * dt;
      if (t > tEnd) break;
      const float phi = sample_phi(f, ro + t * rd);
      if ((phi > 0.5f) != startInWater) {
        const float u = (0.5f - prevPhi) / (phi - prevPhi);
        tSurface = prevT + u * (t - prevT);
        break;
      }
      prevT = t;
      prevPhi = phi;
    }
    if (tSurface > 0.0f) {
      const V3 wpSurf = ro + tSurface * rd;
      V3 n = normalize(grad_phi(f, wpSurf) + v3(1e-6f, 1e-6f, 1e-6f));
      if (startInWater) n = -n;
      if (dot(n, rd) > 0.0f) n = -n;
      const bool entering = !startInWater;
      const float ior = entering ? (1.0f / 1.33f) : (1.33f / 1.0f);
      const V3 reflDir = reflect(rd, n);
      const V3 refrDir = refract(rd, n, ior);
      const bool tir = dot(refrDir, refrDir) < 1e-4f;
      V3 reflCol = sky_color(f, reflDir);
      if (startInWater) reflCol = water_attenuate(reflCol, tSurface - tEnter);
      V3 refrCol;
      if (tir) {
        refrCol = reflCol;
      } else {
        float tBack;
        const V3 back = trace_backdrop(f, wpSurf + 0.003f * refrDir, refrDir, tBack);
        refrCol = entering ? water_attenuate(back, tBack) : water_attenuate(back, tSurface - tEnter);
      }
      const float cosI = fmaxf(dot(-rd, n), 0.0f);
      col = mix(refrCol, reflCol, fresnel_schlick(cosI, 0.02f));
      const V3 h = normalize(-f.light + -rd);
      col = col + v3(1.0f, 0.95f, 0.85f) * (powf(fmaxf(dot(h, n), 0.0f), 256.0f) * 0.6f);
    } else {
      const V3 back = tSphere > 0.0f ? shade_sphere(f, ro + tSphere * rd, rd) : sky_color(f, rd);
      col = startInWater ? water_attenuate(back, tEnd - tEnter) : back;
    }
    col = tonemap(col);
  }
  // RGBA8, top row first
  uint8_t *o = f.out + 4 * ((long long)(f.height - 1 - py) * f.width + px);
  o[0] = (uint8_t)__float2int_rn(clampf(col.x, 0.0f, 1.0f) * 255.0f);
  o[1] = (uint8_t)__float2int_rn(clampf(col.y, 0.0f, 1.0f) * 255.0f);
  o[2] = (uint8_t)__float2int_rn(clampf(col.z, 0.0f, 1.0f) * 255.0f);
  o[3] = 255;
}

}  // namespace

// Camera and matrices as src/render.js builds them: doubles, stored to float
// like its Float32Array matrices and uniform3f values.
void render_frame_setup(int nx, int ny, int nz, const lbm_sphere *sphere, const lbm_camera *cam, int width,
                        int height, RenderSetup *out) {
  const double maxN = (double)std::max(nx, std::max(ny, nz));
  const double box[3] = {nx / maxN, ny / maxN, nz / maxN};
  const double tgt[3] = {box[0] * 0.5, box[1] * 0.5, box[2] * 0.5};
  const double eye[3] = {tgt[0] + cam->dist * cos(cam->elev) * sin(cam->azimuth),
                         tgt[1] - cam->dist * sin(cam->elev),
                         tgt[2] + cam->dist * cos(cam->elev) * cos(cam->azimuth)};
  const double up[3] = {0, -1, 0};
  // perspective (fovy pi/3, near 0.05, far 20)
  float P[16];
  {
    const double aspect = (double)width / (double)height;
    const double fy = 1.0 / tan(M_PI / 3 * 0.5), nf = 1.0 / (0.05 - 20.0);
    const double v[16] = {fy / aspect, 0, 0, 0, 0, fy, 0, 0, 0, 0, (20.0 + 0.05) * nf, -1, 0, 0, 2 * 20.0 * 0.05 * nf, 0};
    for (int i = 0; i < 16; i++) P[i] = (float)v[i];
  }
  // look-at
  float V[16];
  {
    const double z0 = eye[0] - tgt[0], z1 = eye[1] - tgt[1], z2 = eye[2] - tgt[2];
    double zl = sqrt(z0 * z0 + z1 * z1 + z2 * z2);
    if (zl < 1e-9) zl = 1;
    const double zx = z0 / zl, zy = z1 / zl, zz = z2 / zl;
    double xx = up[1] * zz - up[2] * zy, xy = up[2] * zx - up[0] * zz, xz = up[0] * zy - up[1] * zx;
    double xl = sqrt(xx * xx + xy * xy + xz * xz);
    if (xl < 1e-9) xl = 1;
    xx /= xl;
    xy /= xl;
    xz /= xl;
    const double yx = zy * xz - zz * xy, yy = zz * xx - zx * xz, yz = zx * xy - zy * xx;
    const double v[16] = {xx, yx, zx, 0, xy, yy, zy, 0, xz, yz, zz, 0,
                          -(xx * eye[0] + xy * eye[1] + xz * eye[2]),
                          -(yx * eye[0] + yy * eye[1] + yz * eye[2]),
                          -(zx * eye[0] + zy * eye[1] + zz * eye[2]), 1};
    for (int i = 0; i < 16; i++) V[i] = (float)v[i];
  }
  // vp = P * V (column-major), products in double, stored float
  float M[16];
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++)
      M[i * 4 + j] = (float)((double)P[0 * 4 + j] * V[i * 4 + 0] + (double)P[1 * 4 + j] * V[i * 4 + 1] +
                             (double)P[2 * 4 + j] * V[i * 4 + 2] + (double)P[3 * 4 + j] * V[i * 4 + 3]);
  // inverse by cofactors, in double
  {
    const double a00 = M[0], a01 = M[1], a02 = M[2], a03 = M[3], a10 = M[4], a11 = M[5], a12 = M[6],
                 a13 = M[7], a20 = M[8], a21 = M[9], a22 = M[10], a23 = M[11], a30 = M[12], a31 = M[13],
                 a32 = M[14], a33 = M[15];
    const double b00 = a00 * a11 - a01 * a10, b01 = a00 * a12 - a02 * a10, b02 = a00 * a13 - a03 * a10,
                 b03 = a01 * a12 - a02 * a11, b04 = a01 * a13 - a03 * a11, b05 = a02 * a13 - a03 * a12,
                 b06 = a20 * a31 - a21 * a30, b07 = a20 * a32 - a22 * a30, b08 = a20 * a33 - a23 * a30,
                 b09 = a21 * a32 - a22 * a31, b10 = a21 * a33 - a23 * a31, b11 = a22 * a33 - a23 * a32;
    double det = b00 * b11 - b01 * b10 + b02 * b09 + b03 * b08 - b04 * b07 + b05 * b06;
    if (det == 0) {
      for (int i = 0; i < 16; i++) out->inv[i] = (i % 5 == 0) ? 1.0f : 0.0f;
    } else {
      det = 1.0 / det;
      const double r[16] = {(a11 * b11 - a12 * b10 + a13 * b09) * det, (-a01 * b11 + a02 * b10 - a03 * b09) * det,
                            (a31 * b05 - a32 * b04 + a33 * b03) * det, (-a21 * b05 + a22 * b04 - a23 * b03) * det,
                            (-a10 * b11 + a12 * b08 - a13 * b07) * det, (a00 * b11 - a02 * b08 + a03 * b07) * det,
                            (-a30 * b05 + a32 * b02 - a33 * b01) * det, (a20 * b05 - a22 * b02 + a23 * b01) * det,
                            (a10 * b10 - a11 * b08 + a13 * b06) * det, (-a00 * b10 + a01 * b08 - a03 * b06) * det,
                            (a30 * b04 - a31 * b02 + a33 * b00) * det, (-a20 * b04 + a21 * b02 - a23 * b00) * det,
                            (-a10 * b09 + a11 * b07 - a12 * b06) * det, (a00 * b09 - a01 * b07 + a02 * b06) * det,
                            (-a30 * b03 + a31 * b01 - a32 * b00) * det, (a20 * b03 - a21 * b01 + a22 * b00) * det};
      for (int i = 0; i < 16; i++) out->inv[i] = (float)r[i];
    }
  }
  for (int a = 0; a < 3; a++) {
    out->cam[a] = (float)eye[a];
    out->boxMax[a] = (float)box[a];
  }
  out->gridInv[0] = (float)(1.0 / nx);
  out->gridInv[1] = (float)(1.0 / ny);
  out->gridInv[2] = (float)(1.0 / nz);
  const double L = sqrt(cam->light[0] * cam->light[0] + cam->light[1] * cam->light[1] +
                        cam->light[2] * cam->light[2]);
  for (int a = 0; a < 3; a++) out->light[a] = (float)(cam->light[a] / L);
  if (sphere) {
    out->sph[0] = (float)(sphere->cx / maxN);
    out->sph[1] = (float)(sphere->cy / maxN);
    out->sph[2] = (float)(sphere->cz / maxN);
    out->sph[3] = (float)(sphere->r / maxN);
  } else {
    out->sph[0] = out->sph[1] = out->sph[2] = out->sph[3] = 0.0f;
  }
}

cudaError_t render_launch(const uint8_t *d_vol, int nx, int ny, int nz, const RenderSetup &r, int width,
                          int height, uint8_t *d_out, cudaStream_t st) {
  Frame f;
  f.vol = d_vol;
  f.nx = nx;
  f.ny = ny;
  f.nz = nz;
  f.width = width;
  f.height = height;
  memcpy(f.inv, r.inv, sizeof(f.inv));
  f.cam = {r.cam[0], r.cam[1], r.cam[2]};
  f.gridInv = {r.gridInv[0], r.gridInv[1], r.gridInv[2]};
  f.boxMax = {r.boxMax[0], r.boxMax[1], r.boxMax[2]};
  f.light = {r.light[0], r.light[1], r.light[2]};
  f.sphC = {r.sph[0], r.sph[1], r.sph[2]};
  f.sphR = r.sph[3];
  f.out = d_out;
  dim3 block(16, 8);
  dim3 grid((width + 15) / 16, (height + 7) / 8);
  k_render<<<grid, block, 0, st>>>(f);
  return cudaGetLastError();
}

}  // namespace lbm

extern "C" int lbm_render_volume(const uint8_t *d_vol, int nx, int ny, int nz, const lbm_sphere *sphere,
                                 const lbm_camera *cam, int width, int height, uint8_t *d_out, void *stream) {
  if (!d_vol || !d_out || !cam || nx < 1 || ny < 1 || nz < 1 || width < 1 || height < 1 ||
      (long long)width * height > (1LL << 28))
    return LBM_ERR_ARG;
  lbm::RenderSetup r;
  lbm::render_frame_setup(nx, ny, nz, sphere, cam, width, height, &r);
  return lbm::render_launch(d_vol, nx, ny, nz, r, width, height, d_out, (cudaStream_t)stream) == cudaSuccess
             ? LBM_OK
             : LBM_ERR_CUDA;
}

extern "C" void lbm_camera_default(lbm_camera *cam) {
  if (!cam) return;
  cam->azimuth = M_PI * 0.25;
  cam->elev = -0.25;
  cam->dist = 2.4;
  cam->light[0] = 0.35;
  cam->light[1] = 0.75;
  cam->light[2] = 0.5;
}
