/*
 * CPU oracle for the headless renderer -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's WebGL2 renderer (src/render.js):
 * the orbit camera and matrices of class Renderer (src/render.js:273-353,
 * 405-448, 484-513: doubles stored to float, like its Float32Array matrices
 * and uniform3f values) and the fragment shader FS_SRC (src/render.js:19-268)
 * in float arithmetic: AABB and sphere intersection, sky and sphere shading,
 * the 48-step march for the phi = 0.5 crossing with the per-pixel jitter,
 * gradient normal, reflection / refraction with Schlick Fresnel and
 * Beer-Lambert tint, tonemap and gamma.  The RG8 3D texture is sampled with
 * linear filtering and clamp-to-edge (src/render.js:391-399), texel centres at
 * (i + 0.5) / n.  Output RGBA8, top row first (the GL window's row 0 is the
 * bottom).  Built without FMA contraction.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

typedef struct { float x, y, z; } v3;
static v3 mk(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 neg(v3 a) { return mk(-a.x, -a.y, -a.z); }
static v3 mul(v3 a, v3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
static v3 scl(v3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
static v3 dv(v3 a, v3 b) { return mk(a.x / b.x, a.y / b.y, a.z / b.z); }
static float dot3(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static v3 nrm(v3 a) { return scl(a, 1.0f / sqrtf(dot3(a, a))); }
static float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }
static v3 mixv(v3 x, v3 y, float a) { return add(scl(x, 1.0f - a), scl(y, a)); }

typedef struct {
  const uint8_t *vol;
  int nx, ny, nz;
  float inv[16];
  v3 cam, gridInv, boxMax, light, sphC;
  float sphR;
} frame;

static float tex(const frame *f, int x, int y, int z) {
  return (float)f->vol[2 * (((long long)z * f->ny + y) * f->nx + x)] * (1.0f / 255.0f);
}
static int cl(int v, int n) { return v < 0 ? 0 : (v > n - 1 ? n - 1 : v); }

static float sample_phi(const frame *f, v3 wp) {
  v3 uvw = dv(wp, f->boxMax);
  float u = uvw.x * (float)f->nx - 0.5f, v = uvw.y * (float)f->ny - 0.5f, w = uvw.z * (float)f->nz - 0.5f;
  float fu = floorf(u), fv = floorf(v), fw = floorf(w);
  float a = u - fu, b = v - fv, c = w - fw;
  int x0 = (int)fu, y0 = (int)fv, z0 = (int)fw;
  int x1 = cl(x0 + 1, f->nx), y1 = cl(y0 + 1, f->ny), z1 = cl(z0 + 1, f->nz);
  x0 = cl(x0, f->nx);
  y0 = cl(y0, f->ny);
  z0 = cl(z0, f->nz);
  float c00 = tex(f, x0, y0, z0) * (1.0f - a) + tex(f, x1, y0, z0) * a;
  float c10 = tex(f, x0, y1, z0) * (1.0f - a) + tex(f, x1, y1, z0) * a;
  float c01 = tex(f, x0, y0, z1) * (1.0f - a) + tex(f, x1, y0, z1) * a;
  float c11 = tex(f, x0, y1, z1) * (1.0f - a) + tex(f, x1, y1, z1) * a;
  float c0 = c00 * (1.0f - b) + c10 * b;
  float c1 = c01 * (1.0f - b) + c11 * b;
  return c0 * (1.0f - c) + c1 * c;
}

static v3 grad_phi(const frame *f, v3 wp) {
  v3 e = mul(f->boxMax, f->gridInv);
  return mk(sample_phi(f, add(wp, mk(e.x, 0, 0))) - sample_phi(f, sub(wp, mk(e.x, 0, 0))),
            sample_phi(f, add(wp, mk(0, e.y, 0))) - sample_phi(f, sub(wp, mk(0, e.y, 0))),
            sample_phi(f, add(wp, mk(0, 0, e.z))) - sample_phi(f, sub(wp, mk(0, 0, e.z))));
}

static void aabb(v3 ro, v3 rd, v3 bmax, float *tn, float *tf) {
  v3 inv = mk(1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z);
  v3 t1 = mul(sub(mk(0, 0, 0), ro), inv), t2 = mul(sub(bmax, ro), inv);
  v3 lo = mk(fminf(t1.x, t2.x), fminf(t1.y, t2.y), fminf(t1.z, t2.z));
  v3 hi = mk(fmaxf(t1.x, t2.x), fmaxf(t1.y, t2.y), fmaxf(t1.z, t2.z));
  *tn = fmaxf(fmaxf(lo.x, lo.y), lo.z);
  *tf = fminf(fminf(hi.x, hi.y), hi.z);
}

static float sphere_hit(v3 ro, v3 rd, v3 c, float r) {
  v3 oc = sub(ro, c);
  float b = dot3(oc, rd);
  float cc = dot3(oc, oc) - r * r;
  float d = b * b - cc;
  if (d < 0.0f) return -1.0f;
  d = sqrtf(d);
  float t = -b - d;
  if (t < 0.0f) t = -b + d;
  return t;
}

static v3 sky(const frame *f, v3 rd) {
  float t = clampf(-rd.y * 0.5f + 0.5f, 0.0f, 1.0f);
  t = clampf(t, 0.0f, 1.0f);
  float s = t * t * (3.0f - 2.0f * t);
  v3 c = mixv(mk(0.72f, 0.78f, 0.86f), mk(0.18f, 0.32f, 0.55f), s);
  float sun = powf(fmaxf(dot3(rd, neg(f->light)), 0.0f), 96.0f);
  return add(c, scl(mk(1.0f, 0.92f, 0.72f), sun * 0.9f));
}

static v3 shade_sphere(const frame *f, v3 wp, v3 rd) {
  v3 n = nrm(sub(wp, f->sphC));
  float lambert = fmaxf(dot3(n, neg(f->light)), 0.0f);
  v3 col = scl(mk(0.95f, 0.78f, 0.35f), 0.22f + 0.85f * lambert);
  v3 h = nrm(sub(neg(f->light), rd));
  col = add(col, scl(mk(1, 1, 1), powf(fmaxf(dot3(h, n), 0.0f), 48.0f) * 0.55f));
  float rim = powf(1.0f - fmaxf(dot3(neg(rd), n), 0.0f), 3.0f);
  return add(col, scl(mk(1.0f, 0.85f, 0.6f), rim * 0.18f));
}

static v3 backdrop(const frame *f, v3 ro, v3 rd, float *outT) {
  float tn, tf;
  aabb(ro, rd, f->boxMax, &tn, &tf);
  float tExit = fmaxf(tf, 0.0f);
  float tS = sphere_hit(ro, rd, f->sphC, f->sphR);
  if (tS > 0.0f && tS < tExit) {
    *outT = tS;
    return shade_sphere(f, add(ro, scl(rd, tS)), rd);
  }
  *outT = tExit;
  return sky(f, rd);
}

static v3 attenuate(v3 back, float d) {
  v3 tr = mk(expf(-2.6f * d), expf(-0.55f * d), expf(-0.25f * d));
  return add(mul(tr, back), mul(sub(mk(1, 1, 1), tr), mk(0.03f, 0.11f, 0.16f)));
}

static v3 tonemap(v3 c) {
  c = dv(c, add(c, mk(1, 1, 1)));
  return mk(powf(c.x, 1.0f / 2.2f), powf(c.y, 1.0f / 2.2f), powf(c.z, 1.0f / 2.2f));
}

static v3 point(const float *m, float x, float y, float z) {
  float o[4];
  for (int i = 0; i < 4; i++) o[i] = m[i] * x + m[4 + i] * y + m[8 + i] * z + m[12 + i] * 1.0f;
  return mk(o[0] / o[3], o[1] / o[3], o[2] / o[3]);
}

static v3 pixel(const frame *f, int px, int py, int w, int h) {
  float uvx = ((float)px + 0.5f) / (float)w, uvy = ((float)py + 0.5f) / (float)h;
  float ndx = uvx * 2.0f - 1.0f, ndy = uvy * 2.0f - 1.0f;
  v3 wn = point(f->inv, ndx, ndy, -1.0f), wf = point(f->inv, ndx, ndy, 1.0f);
  v3 rd = nrm(sub(wf, wn)), ro = f->cam;
  float tn, tf;
  aabb(ro, rd, f->boxMax, &tn, &tf);
  float tEnter = fmaxf(tn, 0.0f), tExit = tf;
  if (tExit < tEnter) return tonemap(sky(f, rd));
  float tRaw = sphere_hit(ro, rd, f->sphC, f->sphR);
  float tSphere = (tRaw > tEnter && tRaw < tExit) ? tRaw : -1.0f;
  float tEnd = tSphere > 0.0f ? tSphere : tExit;
  float epsT = 0.002f * (tEnd - tEnter);
  float prevT = tEnter + epsT;
  float prevPhi = sample_phi(f, add(ro, scl(rd, prevT)));
  int startIn = prevPhi > 0.5f;
  float dt = (tEnd - prevT) / 48.0f;
  float s = sinf(uvx * 12.9898f + uvy * 78.233f) * 43758.5453f;
  float jit = s - floorf(s);
  float tSurf = -1.0f;
  for (int i = 0; i < 48; i++) {
    float t = prevT + ((float)i + 0.5f + jit) * dt;
    if (t > tEnd) break;
    float phi = sample_phi(f, add(ro, scl(rd, t)));
    if ((phi > 0.5f) != startIn) {
      float u = (0.5f - prevPhi) / (phi - prevPhi);
      tSurf = prevT + u * (t - prevT);
      break;
    }
    prevT = t;
    prevPhi = phi;
  }
  v3 col;
  if (tSurf > 0.0f) {
    v3 wp = add(ro, scl(rd, tSurf));
    v3 n = nrm(add(grad_phi(f, wp), mk(1e-6f, 1e-6f, 1e-6f)));
    if (startIn) n = neg(n);
    if (dot3(n, rd) > 0.0f) n = neg(n);
    int entering = !startIn;
    float eta = entering ? (1.0f / 1.33f) : (1.33f / 1.0f);
    v3 refl = sub(rd, scl(n, 2.0f * dot3(n, rd)));
    float d = dot3(n, rd);
    float k = 1.0f - eta * eta * (1.0f - d * d);
    v3 refr = k < 0.0f ? mk(0, 0, 0) : sub(scl(rd, eta), scl(n, eta * d + sqrtf(k)));
    int tir = dot3(refr, refr) < 1e-4f;
    v3 reflCol = sky(f, refl);
    if (startIn) reflCol = attenuate(reflCol, tSurf - tEnter);
    v3 refrCol;
    if (tir) {
      refrCol = reflCol;
    } else {
      float tBack;
      v3 back = backdrop(f, add(wp, scl(refr, 0.003f)), refr, &tBack);
      refrCol = entering ? attenuate(back, tBack) : attenuate(back, tSurf - tEnter);
    }
    float cosI = fmaxf(dot3(neg(rd), n), 0.0f);
    float fres = 0.02f + (1.0f - 0.02f) * powf(1.0f - cosI, 5.0f);
    col = mixv(refrCol, reflCol, fres);
    v3 hh = nrm(add(neg(f->light), neg(rd)));
    col = add(col, scl(mk(1.0f, 0.95f, 0.85f), powf(fmaxf(dot3(hh, n), 0.0f), 256.0f) * 0.6f));
  } else {
    v3 back = tSphere > 0.0f ? shade_sphere(f, add(ro, scl(rd, tSphere)), rd) : sky(f, rd);
    col = startIn ? attenuate(back, tEnd - tEnter) : back;
  }
  return tonemap(col);
}

/* sphere: cx, cy, cz, r in cells, or NULL; cam: azimuth, elev, dist, light[3] */
void or_render(const uint8_t *vol, int nx, int ny, int nz, const double *sphere, const double *cam, int w,
               int h, uint8_t *out) {
  double maxN = nx > ny ? nx : ny;
  if (nz > maxN) maxN = nz;
  double box[3] = {nx / maxN, ny / maxN, nz / maxN};
  double tg[3] = {box[0] * 0.5, box[1] * 0.5, box[2] * 0.5};
  double az = cam[0], el = cam[1], dist = cam[2];
  double eye[3] = {tg[0] + dist * cos(el) * sin(az), tg[1] - dist * sin(el), tg[2] + dist * cos(el) * cos(az)};
  double up[3] = {0, -1, 0};
  float P[16], V[16], M[16], I[16];
  double aspect = (double)w / (double)h;
  double fy = 1.0 / tan(M_PI / 3 * 0.5), nf = 1.0 / (0.05 - 20.0);
  double pv[16] = {fy / aspect, 0, 0, 0, 0, fy, 0, 0, 0, 0, (20.0 + 0.05) * nf, -1, 0, 0, 2 * 20.0 * 0.05 * nf, 0};
  for (int i = 0; i < 16; i++) P[i] = (float)pv[i];
  double z0 = eye[0] - tg[0], z1 = eye[1] - tg[1], z2 = eye[2] - tg[2];
  double zl = sqrt(z0 * z0 + z1 * z1 + z2 * z2);
  if (zl < 1e-9) zl = 1;
  double zx = z0 / zl, zy = z1 / zl, zz = z2 / zl;
  double xx = up[1] * zz - up[2] * zy, xy = up[2] * zx - up[0] * zz, xz = up[0] * zy - up[1] * zx;
  double xl = sqrt(xx * xx + xy * xy + xz * xz);
  if (xl < 1e-9) xl = 1;
  xx /= xl;
  xy /= xl;
  xz /= xl;
  double yx = zy * xz - zz * xy, yy = zz * xx - zx * xz, yz = zx * xy - zy * xx;
  double vv[16] = {xx, yx, zx, 0, xy, yy, zy, 0, xz, yz, zz, 0, -(xx * eye[0] + xy * eye[1] + xz * eye[2]),
                   -(yx * eye[0] + yy * eye[1] + yz * eye[2]), -(zx * eye[0] + zy * eye[1] + zz * eye[2]), 1};
  for (int i = 0; i < 16; i++) V[i] = (float)vv[i];
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++)
      M[i * 4 + j] = (float)((double)P[j] * V[i * 4] + (double)P[4 + j] * V[i * 4 + 1] +
                             (double)P[8 + j] * V[i * 4 + 2] + (double)P[12 + j] * V[i * 4 + 3]);
  {
    double a00 = M[0], a01 = M[1], a02 = M[2], a03 = M[3], a10 = M[4], a11 = M[5], a12 = M[6], a13 = M[7];
    double a20 = M[8], a21 = M[9], a22 = M[10], a23 = M[11], a30 = M[12], a31 = M[13], a32 = M[14], a33 = M[15];
    double b00 = a00 * a11 - a01 * a10, b01 = a00 * a12 - a02 * a10, b02 = a00 * a13 - a03 * a10;
    double b03 = a01 * a12 - a02 * a11, b04 = a01 * a13 - a03 * a11, b05 = a02 * a13 - a03 * a12;
    double b06 = a20 * a31 - a21 * a30, b07 = a20 * a32 - a22 * a30, b08 = a20 * a33 - a23 * a30;
    double b09 = a21 * a32 - a22 * a31, b10 = a21 * a33 - a23 * a31, b11 = a22 * a33 - a23 * a32;
    double det = b00 * b11 - b01 * b10 + b02 * b09 + b03 * b08 - b04 * b07 + b05 * b06;
    if (det == 0) {
      for (int i = 0; i < 16; i++) I[i] = (i % 5 == 0) ? 1.0f : 0.0f;
    } else {
      det = 1.0 / det;
      double r[16] = {(a11 * b11 - a12 * b10 + a13 * b09) * det, (-a01 * b11 + a02 * b10 - a03 * b09) * det,
                      (a31 * b05 - a32 * b04 + a33 * b03) * det, (-a21 * b05 + a22 * b04 - a23 * b03) * det,
                      (-a10 * b11 + a12 * b08 - a13 * b07) * det, (a00 * b11 - a02 * b08 + a03 * b07) * det,
                      (-a30 * b05 + a32 * b02 - a33 * b01) * det, (a20 * b05 - a22 * b02 + a23 * b01) * det,
                      (a10 * b10 - a11 * b08 + a13 * b06) * det, (-a00 * b10 + a01 * b08 - a03 * b06) * det,
                      (a30 * b04 - a31 * b02 + a33 * b00) * det, (-a20 * b04 + a21 * b02 - a23 * b00) * det,
                      (-a10 * b09 + a11 * b07 - a12 * b06) * det, (a00 * b09 - a01 * b07 + a02 * b06) * det,
                      (-a30 * b03 + a31 * b01 - a32 * b00) * det, (a20 * b03 - a21 * b01 + a22 * b00) * det};
      for (int i = 0; i < 16; i++) I[i] = (float)r[i];
    }
  }
  frame f;
  f.vol = vol;
  f.nx = nx;
  f.ny = ny;
  f.nz = nz;
  memcpy(f.inv, I, sizeof(I));
  f.cam = mk((float)eye[0], (float)eye[1], (float)eye[2]);
  f.gridInv = mk((float)(1.0 / nx), (float)(1.0 / ny), (float)(1.0 / nz));
  f.boxMax = mk((float)box[0], (float)box[1], (float)box[2]);
  double L = sqrt(cam[3] * cam[3] + cam[4] * cam[4] + cam[5] * cam[5]);
  f.light = mk((float)(cam[3] / L), (float)(cam[4] / L), (float)(cam[5] / L));
  if (sphere) {
    f.sphC = mk((float)(sphere[0] / maxN), (float)(sphere[1] / maxN), (float)(sphere[2] / maxN));
    f.sphR = (float)(sphere[3] / maxN);
  } else {
    f.sphC = mk(0, 0, 0);
    f.sphR = 0.0f;
  }
  for (int py = 0; py < h; py++)
    for (int px = 0; px < w; px++) {
      v3 c = pixel(&f, px, py, w, h);
      uint8_t *o = out + 4 * ((long long)(h - 1 - py) * w + px);
      o[0] = (uint8_t)lrintf(clampf(c.x, 0.0f, 1.0f) * 255.0f);
      o[1] = (uint8_t)lrintf(clampf(c.y, 0.0f, 1.0f) * 255.0f);
      o[2] = (uint8_t)lrintf(clampf(c.z, 0.0f, 1.0f) * 255.0f);
      o[3] = 255;
    }
}
