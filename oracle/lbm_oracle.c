/*
 * CPU oracle for the LBM step -- TEST INFRASTRUCTURE ONLY (see lbm_oracle.h).
 *
 * Restates src/lattices.js, src/sim.js and src/solid.js of the reference with
 * JavaScript number semantics: double intermediates, float32 rounding only on
 * stores into Float32Array fields, left-to-right evaluation, no contraction.
 * Each function cites the reference lines it follows.
 */
#include "lbm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ---------------------------------------------------------------- tables */
/* src/lattices.js:34-49 (D3Q27 in opposite pairs), 52-57 (weights),
 * 66-69 (OPP = k^1 pairing), 79-91 (D3Q7). */
static int8_t EX27[27], EY27[27], EZ27[27], OPP27[27];
static float W27[27];
static int8_t EX7[7], EY7[7], EZ7[7], OPP7[7];
static float W7[7];
static int tables_ready = 0;

static void build_tables(void) {
  if (tables_ready) return;
  /* rest, 6 faces, 12 edges, 8 corners; consecutive entries are opposites */
  static const int8_t d[27][3] = {
      {0, 0, 0},   {1, 0, 0},  {-1, 0, 0},  {0, 1, 0},   {0, -1, 0}, {0, 0, 1},
      {0, 0, -1},  {1, 1, 0},  {-1, -1, 0}, {1, -1, 0},  {-1, 1, 0}, {1, 0, 1},
      {-1, 0, -1}, {1, 0, -1}, {-1, 0, 1},  {0, 1, 1},   {0, -1, -1}, {0, 1, -1},
      {0, -1, 1},  {1, 1, 1},  {-1, -1, -1}, {1, 1, -1}, {-1, -1, 1}, {1, -1, 1},
      {-1, 1, -1}, {-1, 1, 1}, {1, -1, -1}};
  for (int k = 0; k < 27; k++) {
    EX27[k] = d[k][0];
    EY27[k] = d[k][1];
    EZ27[k] = d[k][2];
    int nz = (d[k][0] != 0) + (d[k][1] != 0) + (d[k][2] != 0);
    double w = nz == 0 ? 8.0 / 27.0 : nz == 1 ? 2.0 / 27.0 : nz == 2 ? 1.0 / 54.0 : 1.0 / 216.0;
    W27[k] = (float)w; /* Float32Array store */
    OPP27[k] = k == 0 ? 0 : ((k & 1) ? k + 1 : k - 1);
  }
  for (int k = 0; k < 7; k++) {
    EX7[k] = d[k][0];
    EY7[k] = d[k][1];
    EZ7[k] = d[k][2];
    W7[k] = (float)(k == 0 ? 0.25 : 0.125);
    OPP7[k] = k == 0 ? 0 : ((k & 1) ? k + 1 : k - 1);
  }
  tables_ready = 1;
}

void or_tables(int8_t ex27[27], int8_t ey27[27], int8_t ez27[27], float w27[27],
               int8_t opp27[27], int8_t ex7[7], int8_t ey7[7], int8_t ez7[7],
               float w7[7], int8_t opp7[7]) {
  build_tables();
  memcpy(ex27, EX27, 27);
  memcpy(ey27, EY27, 27);
  memcpy(ez27, EZ27, 27);
  memcpy(w27, W27, sizeof(W27));
  memcpy(opp27, OPP27, 27);
  memcpy(ex7, EX7, 7);
  memcpy(ey7, EY7, 7);
  memcpy(ez7, EZ7, 7);
  memcpy(w7, W7, sizeof(W7));
  memcpy(opp7, OPP7, 7);
}

/* src/lattices.js:95-99 */
#define INV_CS2_27 3.0
#define INV_2CS4_27 4.5
#define CS2_7 0.25
#define INV_CS2_7 4.0

int or_store_bytes(void) { return (int)sizeof(or_real); }

/* ---------------------------------------------------------------- create */
/* src/sim.js:30-96 */
or_sim *or_sim_create(int nx, int ny, int nz) {
  build_tables();
  or_sim *s = (or_sim *)calloc(1, sizeof(or_sim));
  s->nx = nx;
  s->ny = ny;
  s->nz = nz;
  int n = nx * ny * nz;
  s->n = n;
  s->f = (or_real *)calloc((size_t)n * 27, sizeof(or_real));
  s->f2 = (or_real *)calloc((size_t)n * 27, sizeof(or_real));
  s->h = (or_real *)calloc((size_t)n * 7, sizeof(or_real));
  s->h2 = (or_real *)calloc((size_t)n * 7, sizeof(or_real));
  or_real **scalars[] = {&s->rho, &s->ux, &s->uy, &s->uz, &s->phi, &s->phiPrev,
                       &s->usx, &s->usy, &s->usz, &s->gx, &s->gy, &s->gz,
                       &s->lap, &s->bodyFx, &s->bodyFy, &s->bodyFz};
  for (size_t a = 0; a < sizeof(scalars) / sizeof(scalars[0]); a++)
    *scalars[a] = (or_real *)calloc((size_t)n, sizeof(or_real));
  s->tag = (uint8_t *)calloc((size_t)n, 1);
  s->tagPrev = (uint8_t *)calloc((size_t)n, 1);
  int nxny = nx * ny;
  for (int k = 0; k < 27; k++) {
    int off = -(EZ27[k] * nxny + EY27[k] * nx + EX27[k]);
    s->neighOffset27[k] = off;
    s->fOffset27[k] = off * 27 + k;
  }
  for (int k = 0; k < 7; k++) {
    int off = -(EZ7[k] * nxny + EY7[k] * nx + EX7[k]);
    s->neighOffset7[k] = off;
    s->hOffset7[k] = off * 7 + k;
  }
  s->tau = 0.6;
  s->tauPhi = 0.7;
  s->sigma = 0.012;
  s->gravity = 0.0010;
  s->rhoL = 1.0;
  s->rhoG = 0.05;
  s->W = 4.0;
  s->mobility = 0.02;
  s->omp = 0;
  return s;
}

void or_sim_destroy(or_sim *s) {
  if (!s) return;
  or_real *arrs[] = {s->f, s->f2, s->h, s->h2, s->rho, s->ux, s->uy, s->uz, s->phi,
                   s->phiPrev, s->usx, s->usy, s->usz, s->gx, s->gy, s->gz, s->lap,
                   s->bodyFx, s->bodyFy, s->bodyFz};
  for (size_t a = 0; a < sizeof(arrs) / sizeof(arrs[0]); a++) free(arrs[a]);
  free(s->tag);
  free(s->tagPrev);
  free(s);
}

void or_sim_set_omp(or_sim *s, int nthreads) {
  s->omp = nthreads;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
}

#define IDX(s, x, y, z) ((((z) * (s)->ny) + (y)) * (s)->nx + (x))

/* ---------------------------------------------------------------- init */
/* src/sim.js:112-134 */
void or_init_flat(or_sim *s, double waterlineY) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  const double W = s->W;
  for (int z = 0; z < nz; z++) {
    for (int y = 0; y < ny; y++) {
      double phiCol = 0.5 * (1 + tanh(2 * ((double)y - waterlineY) / W));
      for (int x = 0; x < nx; x++) {
        int i = IDX(s, x, y, z);
        s->phi[i] = (or_real)phiCol;
        s->phiPrev[i] = (or_real)phiCol;
        s->rho[i] = 1.0;
        s->ux[i] = s->uy[i] = s->uz[i] = 0.0;
        int onWall = x == 0 || x == nx - 1 || y == 0 || y == ny - 1 || z == 0 || z == nz - 1;
        s->tag[i] = onWall ? OR_TAG_WALL : OR_TAG_FLUID;
        s->tagPrev[i] = s->tag[i];
        for (int k = 0; k < 27; k++) s->f[(size_t)i * 27 + k] = W27[k];
        for (int k = 0; k < 7; k++) s->h[(size_t)i * 7 + k] = (or_real)((double)W7[k] * phiCol);
      }
    }
  }
  or_seed_hydrostatic(s);
}

/* src/sim.js:144-173: column-wise hydrostatic sum-f with the Guo lattice
 * velocity offset u_lat = (0, -g/2, 0).  Sequential in y per (z, x) column. */
void or_seed_hydrostatic(or_sim *s) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  const double dRho = s->rhoL - s->rhoG;
  const double gOverCs2 = s->gravity * INV_CS2_27;
  const double uLatY = -0.5 * s->gravity;
  const double uLat2 = uLatY * uLatY;
  for (int z = 0; z < nz; z++) {
    for (int x = 0; x < nx; x++) {
      double pCs2 = 1.0;
      for (int y = 0; y < ny; y++) {
        int i = IDX(s, x, y, z);
        s->rho[i] = (or_real)pCs2;
        size_t i27 = (size_t)i * 27;
        double rhoPhase = s->rhoG + (double)s->phi[i] * dRho;
        for (int k = 0; k < 27; k++) {
          double eu = EY27[k] * uLatY;
          double Qi = eu * (INV_CS2_27 + INV_2CS4_27 * eu) - 1.5 * uLat2;
          s->f[i27 + k] = (or_real)((double)W27[k] * (pCs2 + rhoPhase * Qi));
        }
        pCs2 += rhoPhase * gOverCs2;
      }
    }
  }
}

/* ---------------------------------------------------------------- gradients */
/* src/sim.js:176-199: central differences with index clamping at the edges. */
void or_compute_phi_gradients(or_sim *s) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  const or_real *phi = s->phi;
#pragma omp parallel for schedule(static) if (s->omp > 0)
  for (int z = 0; z < nz; z++) {
    int zm = z > 0 ? z - 1 : z, zp = z < nz - 1 ? z + 1 : z;
    for (int y = 0; y < ny; y++) {
      int ym = y > 0 ? y - 1 : y, yp = y < ny - 1 ? y + 1 : y;
      for (int x = 0; x < nx; x++) {
        int xm = x > 0 ? x - 1 : x, xp = x < nx - 1 ? x + 1 : x;
        int i = ((z * ny) + y) * nx + x;
        double c = phi[i];
        double px = phi[((z * ny) + y) * nx + xp];
        double mx = phi[((z * ny) + y) * nx + xm];
        double py = phi[((z * ny) + yp) * nx + x];
        double my = phi[((z * ny) + ym) * nx + x];
        double pz = phi[((zp * ny) + y) * nx + x];
        double mz = phi[((zm * ny) + y) * nx + x];
        s->gx[i] = (or_real)(0.5 * (px - mx));
        s->gy[i] = (or_real)(0.5 * (py - my));
        s->gz[i] = (or_real)(0.5 * (pz - mz));
        s->lap[i] = (or_real)(px + mx + py + my + pz + mz - 6 * c);
      }
    }
  }
}

/* ---------------------------------------------------------------- solids */
/* Composite-solid owner: the first sphere (lowest index) that contains the
 * cell; -1 when none does.  src/solid.js:50-55 for the containment test. */
static int owner_of(const or_sphere *solids, int nsolids, int x, int y, int z) {
  for (int b = 0; b < nsolids; b++)
    if (or_sphere_contains(&solids[b], x, y, z)) return b;
  return -1;
}

/* src/sim.js:214-244 */
void or_retag_cells(or_sim *s, const or_sphere *solids, int nsolids) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  memcpy(s->tagPrev, s->tag, (size_t)s->n);
  memcpy(s->phiPrev, s->phi, (size_t)s->n * sizeof(or_real));
  double tmp[3];
  for (int z = 0; z < nz; z++) {
    int zOnWall = z == 0 || z == nz - 1;
    for (int y = 0; y < ny; y++) {
      int yOnWall = y == 0 || y == ny - 1;
      for (int x = 0; x < nx; x++) {
        int i = IDX(s, x, y, z);
        if (zOnWall || yOnWall || x == 0 || x == nx - 1) {
          s->tag[i] = OR_TAG_WALL;
          s->usx[i] = s->usy[i] = s->usz[i] = 0.0;
          continue;
        }
        int b = solids ? owner_of(solids, nsolids, x, y, z) : -1;
        if (b >= 0) {
          s->tag[i] = OR_TAG_SOLID;
          or_sphere_surface_velocity(&solids[b], x, y, z, tmp);
          s->usx[i] = (or_real)tmp[0];
          s->usy[i] = (or_real)tmp[1];
          s->usz[i] = (or_real)tmp[2];
        } else {
          s->tag[i] = OR_TAG_FLUID;
          s->usx[i] = s->usy[i] = s->usz[i] = 0.0;
        }
      }
    }
  }
}

/* src/sim.js:257-310: in-place, scan-order-dependent reseeding of cells that
 * switched SOLID -> FLUID (later fresh cells see earlier ones' new values). */
void or_handle_fresh_cells(or_sim *s) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  for (int z = 1; z < nz - 1; z++) {
    for (int y = 1; y < ny - 1; y++) {
      for (int x = 1; x < nx - 1; x++) {
        int i = ((z * ny) + y) * nx + x;
        if (s->tag[i] != OR_TAG_FLUID || s->tagPrev[i] != OR_TAG_SOLID) continue;
        double psum = 0, rsum = 0, vxs = 0, vys = 0, vzs = 0;
        int pcnt = 0;
        for (int dz = -1; dz <= 1; dz++)
          for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++) {
              if (!dx && !dy && !dz) continue;
              int j = (((z + dz) * ny) + (y + dy)) * nx + (x + dx);
              if (s->tag[j] == OR_TAG_FLUID) {
                psum += s->phi[j];
                rsum += s->rho[j];
                vxs += s->ux[j];
                vys += s->uy[j];
                vzs += s->uz[j];
                pcnt++;
              }
            }
        double p = pcnt > 0 ? psum / pcnt : (double)s->phiPrev[i];
        double r = pcnt > 0 ? rsum / pcnt : 1.0;
        double vx = pcnt > 0 ? vxs / pcnt : 0;
        double vy = pcnt > 0 ? vys / pcnt : 0;
        double vz = pcnt > 0 ? vzs / pcnt : 0;
        s->phi[i] = (or_real)p;
        s->phiPrev[i] = (or_real)p;
        s->rho[i] = (or_real)r;
        s->ux[i] = (or_real)vx;
        s->uy[i] = (or_real)vy;
        s->uz[i] = (or_real)vz;
        double rhoPhase = s->rhoG + p * (s->rhoL - s->rhoG);
        double u2 = vx * vx + vy * vy + vz * vz;
        for (int k = 0; k < 27; k++) {
          double eu = EX27[k] * vx + EY27[k] * vy + EZ27[k] * vz;
          double Qi = eu * (INV_CS2_27 + INV_2CS4_27 * eu) - 1.5 * u2;
          s->f[(size_t)i * 27 + k] = (or_real)((double)W27[k] * (r + rhoPhase * Qi));
        }
        for (int k = 0; k < 7; k++) {
          double eu = EX7[k] * vx + EY7[k] * vy + EZ7[k] * vz;
          s->h[(size_t)i * 7 + k] = (or_real)((double)W7[k] * p * (1 + INV_CS2_7 * eu));
        }
      }
    }
  }
}

/* ---------------------------------------------------------------- phase lattice */
/* src/sim.js:324-364: D3Q7 Allen-Cahn BGK with the interface-sharpening source. */
void or_collide_phase(or_sim *s) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  const double invTau = 1 / s->tauPhi;
  const double Mphi = CS2_7 * (s->tauPhi - 0.5);
  const double guoHalf = 1.0 - 0.5 * invTau;
  const double sharpC = 4.0 * Mphi * guoHalf / s->W;
  const double sharpFac = INV_CS2_7;
#pragma omp parallel for schedule(static) if (s->omp > 0)
  for (int z = 1; z < nz - 1; z++) {
    for (int y = 1; y < ny - 1; y++) {
      for (int x = 1; x < nx - 1; x++) {
        int i = IDX(s, x, y, z);
        if (s->tag[i] != OR_TAG_FLUID) continue;
        size_t i7 = (size_t)i * 7;
        double p = s->phi[i];
        double uxi = s->ux[i], uyi = s->uy[i], uzi = s->uz[i];
        double ggx = s->gx[i], ggy = s->gy[i], ggz = s->gz[i];
        double gmag = sqrt(ggx * ggx + ggy * ggy + ggz * ggz) + 1e-12;
        double sharpen = sharpC * p * (1 - p);
        double Sx = sharpen * sharpFac * ggx / gmag;
        double Sy = sharpen * sharpFac * ggy / gmag;
        double Sz = sharpen * sharpFac * ggz / gmag;
        for (int k = 0; k < 7; k++) {
          double wk = W7[k];
          double eu = EX7[k] * uxi + EY7[k] * uyi + EZ7[k] * uzi;
          double heq = wk * p * (1 + INV_CS2_7 * eu);
          double Fk = wk * (EX7[k] * Sx + EY7[k] * Sy + EZ7[k] * Sz);
          double hk = s->h[i7 + k];
          s->h2[i7 + k] = (or_real)(hk - invTau * (hk - heq) + Fk);
        }
      }
    }
  }
}

/* src/sim.js:376-397: pull stream of h with plain bounce-back. */
void or_stream_phase(or_sim *s) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
#pragma omp parallel for schedule(static) if (s->omp > 0)
  for (int z = 1; z < nz - 1; z++) {
    for (int y = 1; y < ny - 1; y++) {
      for (int x = 1; x < nx - 1; x++) {
        int i = IDX(s, x, y, z);
        if (s->tag[i] != OR_TAG_FLUID) continue;
        size_t i7 = (size_t)i * 7;
        for (int k = 0; k < 7; k++) {
          int sIdx = i + s->neighOffset7[k];
          s->h[i7 + k] = s->tag[sIdx] == OR_TAG_FLUID ? s->h2[(long)i7 + s->hOffset7[k]]
                                                      : s->h2[i7 + OPP7[k]];
        }
      }
    }
  }
}

/* ---------------------------------------------------------------- hydro lattice */
/* src/sim.js:406-464: variable-density (HCZ) BGK with Guo forcing, surface
 * tension mu*grad(phi) and density-aware gravity. */
void or_collide_hydro(or_sim *s) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  const double invTau = 1 / s->tau;
  const double beta = 12 * s->sigma / s->W;
  const double kappa = 1.5 * s->sigma * s->W;
  const double dRho = s->rhoL - s->rhoG;
  const double A = (1 - 0.5 * invTau) * INV_CS2_27;
  const double gravity = s->gravity, rhoG = s->rhoG;
#pragma omp parallel for schedule(static) if (s->omp > 0)
  for (int z = 1; z < nz - 1; z++) {
    for (int y = 1; y < ny - 1; y++) {
      for (int x = 1; x < nx - 1; x++) {
        int i = IDX(s, x, y, z);
        if (s->tag[i] != OR_TAG_FLUID) continue;
        size_t i27 = (size_t)i * 27;
        double sumF = s->rho[i];
        double p = s->phi[i];
        double rhoPhase = rhoG + p * dRho;
        double mu = 4 * beta * p * (p - 1) * (2 * p - 1) - kappa * (double)s->lap[i];
        double fx = (double)s->bodyFx[i] + mu * (double)s->gx[i];
        double fy = (double)s->bodyFy[i] + mu * (double)s->gy[i] + rhoPhase * gravity;
        double fz = (double)s->bodyFz[i] + mu * (double)s->gz[i];
        double uxe = s->ux[i], uye = s->uy[i], uze = s->uz[i];
        double u2 = uxe * uxe + uye * uye + uze * uze;
        double negU2half = -1.5 * u2;
        double uF = uxe * fx + uye * fy + uze * fz;
        for (int k = 0; k < 27; k++) {
          double wk = W27[k];
          double eu = EX27[k] * uxe + EY27[k] * uye + EZ27[k] * uze;
          double Qi = negU2half + eu * (INV_CS2_27 + INV_2CS4_27 * eu);
          double feq = wk * (sumF + rhoPhase * Qi);
          double ekF = EX27[k] * fx + EY27[k] * fy + EZ27[k] * fz;
          double Sk = A * wk * (ekF * (1 + INV_CS2_27 * eu) - uF);
          double fk = s->f[i27 + k];
          s->f2[i27 + k] = (or_real)(fk - invTau * (fk - feq) + Sk);
        }
      }
    }
  }
}

/* src/sim.js:484-582: pull stream of f with halfway bounce-back, Ladd
 * moving-wall correction, momentum exchange into the solid, and the macro
 * update (rho = max(sum f, 0.01), phi = clamp01(sum h), u with the half-force
 * shift and a 0.2 Mach clamp).  Impulses are applied in scan order. */
void or_stream_hydro_and_macro(or_sim *s, or_sphere *solids, int nsolids) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  const double beta = 12 * s->sigma / s->W;
  const double kappa = 1.5 * s->sigma * s->W;
  const double dRho = s->rhoL - s->rhoG;
  const double gravity = s->gravity, rhoG = s->rhoG;
  const int serial = (solids != NULL && nsolids > 0) || s->omp <= 0;
#pragma omp parallel for schedule(static) if (!serial)
  for (int z = 1; z < nz - 1; z++) {
    for (int y = 1; y < ny - 1; y++) {
      for (int x = 1; x < nx - 1; x++) {
        int i = IDX(s, x, y, z);
        if (s->tag[i] != OR_TAG_FLUID) continue;
        size_t i27 = (size_t)i * 27;
        double rhoPhaseOld = rhoG + (double)s->phi[i] * dRho;
        double pSumF = 0, mx = 0, my = 0, mz = 0;
        for (int k = 0; k < 27; k++) {
          int sIdx = i + s->neighOffset27[k];
          int sTag = s->tag[sIdx];
          int ekx = EX27[k], eky = EY27[k], ekz = EZ27[k];
          double fk;
          if (sTag == OR_TAG_FLUID) {
            fk = s->f2[(long)i27 + s->fOffset27[k]];
          } else {
            double fopp = s->f2[i27 + OPP27[k]];
            double corr = 0;
            if (sTag == OR_TAG_SOLID) {
              double eu = ekx * (double)s->usx[sIdx] + eky * (double)s->usy[sIdx] +
                          ekz * (double)s->usz[sIdx];
              corr = 2 * (double)W27[k] * rhoPhaseOld * eu * INV_CS2_27;
            }
            fk = fopp + corr;
            if (sTag == OR_TAG_SOLID && solids && nsolids > 0) {
              double m = fopp + fk;
              int sx = x - ekx, sy = y - eky, sz = z - ekz;
              int b = owner_of(solids, nsolids, sx, sy, sz);
              if (b >= 0) or_sphere_apply_impulse(&solids[b], sx, sy, sz, -m * ekx, -m * eky, -m * ekz);
            }
          }
          s->f[i27 + k] = (or_real)fk;
          pSumF += fk;
          mx += ekx * fk;
          my += eky * fk;
          mz += ekz * fk;
        }
        s->rho[i] = (or_real)(pSumF > 0.01 ? pSumF : 0.01);
        double phiSum = 0;
        for (int k = 0; k < 7; k++) phiSum += s->h[(size_t)i * 7 + k];
        double p = phiSum < 0 ? 0 : phiSum > 1 ? 1 : phiSum;
        s->phi[i] = (or_real)p;
        double rhoPhaseNew = rhoG + p * dRho;
        double mu = 4 * beta * p * (p - 1) * (2 * p - 1) - kappa * (double)s->lap[i];
        double fx = (double)s->bodyFx[i] + mu * (double)s->gx[i];
        double fy = (double)s->bodyFy[i] + mu * (double)s->gy[i] + rhoPhaseNew * gravity;
        double fz = (double)s->bodyFz[i] + mu * (double)s->gz[i];
        double invRho = 1 / rhoPhaseNew;
        double uxn = (mx + 0.5 * fx) * invRho;
        double uyn = (my + 0.5 * fy) * invRho;
        double uzn = (mz + 0.5 * fz) * invRho;
        double u2 = uxn * uxn + uyn * uyn + uzn * uzn;
        const double UMAX = 0.2, UMAX2 = UMAX * UMAX;
        if (u2 > UMAX2) {
          double sc = UMAX / sqrt(u2);
          uxn *= sc;
          uyn *= sc;
          uzn *= sc;
        }
        s->ux[i] = (or_real)uxn;
        s->uy[i] = (or_real)uyn;
        s->uz[i] = (or_real)uzn;
      }
    }
  }
  memset(s->bodyFx, 0, (size_t)s->n * sizeof(or_real));
  memset(s->bodyFy, 0, (size_t)s->n * sizeof(or_real));
  memset(s->bodyFz, 0, (size_t)s->n * sizeof(or_real));
}

/* src/sim.js:202-210 */
void or_step(or_sim *s, or_sphere *solids, int nsolids) {
  or_retag_cells(s, solids, nsolids);
  or_handle_fresh_cells(s);
  or_compute_phi_gradients(s);
  or_collide_phase(s);
  or_stream_phase(s);
  or_collide_hydro(s);
  or_stream_hydro_and_macro(s, solids, nsolids);
}

/* src/sim.js:586-600: R = (clamp01(phi)*255)|0 (truncation; NaN -> 0),
 * G = 255 for SOLID cells only. */
void or_pack_volume(const or_sim *s, uint8_t *out) {
  size_t o = 0;
  for (int i = 0; i < s->n; i++) {
    double p = s->phi[i];
    if (p < 0) p = 0;
    else if (p > 1) p = 1;
    double v = p * 255;
    out[o++] = (uint8_t)(v == v ? (int)v : 0);
    out[o++] = s->tag[i] == OR_TAG_SOLID ? 255 : 0;
  }
}

/* ---------------------------------------------------------------- RigidSphere */
/* src/solid.js:9-37 */
void or_sphere_init(or_sphere *b, int nx, int ny, int nz, double cx, double cy,
                    double cz, double r, double density) {
  memset(b, 0, sizeof(*b));
  b->nx = nx;
  b->ny = ny;
  b->nz = nz;
  b->cx = cx;
  b->cy = cy;
  b->cz = cz;
  b->r = r;
  b->density = density;
  or_sphere_recompute_mass(b);
}

/* src/solid.js:39-44 */
void or_sphere_recompute_mass(or_sphere *b) {
  double V = (4.0 / 3.0) * M_PI * b->r * b->r * b->r;
  b->volume = V;
  b->mass = b->density * V;
  b->I = (2.0 / 5.0) * b->mass * b->r * b->r;
}

/* src/solid.js:50-55 */
int or_sphere_contains(const or_sphere *b, int x, int y, int z) {
  double dx = x + 0.5 - b->cx;
  double dy = y + 0.5 - b->cy;
  double dz = z + 0.5 - b->cz;
  return dx * dx + dy * dy + dz * dz <= b->r * b->r;
}

/* src/solid.js:57-66 */
void or_sphere_surface_velocity(const or_sphere *b, int x, int y, int z, double out[3]) {
  double rx = x + 0.5 - b->cx;
  double ry = y + 0.5 - b->cy;
  double rz = z + 0.5 - b->cz;
  out[0] = b->vx + (b->wy * rz - b->wz * ry);
  out[1] = b->vy + (b->wz * rx - b->wx * rz);
  out[2] = b->vz + (b->wx * ry - b->wy * rx);
}

/* src/solid.js:70-80 */
void or_sphere_apply_impulse(or_sphere *b, int x, int y, int z, double px, double py,
                             double pz) {
  b->Fx += px;
  b->Fy += py;
  b->Fz += pz;
  double rx = x + 0.5 - b->cx;
  double ry = y + 0.5 - b->cy;
  double rz = z + 0.5 - b->cz;
  b->Tx += ry * pz - rz * py;
  b->Ty += rz * px - rx * pz;
  b->Tz += rx * py - ry * px;
}

/* src/solid.js:87-101 (impulses go to the owner sphere of each dead cell). */
void or_absorb_dead_cells(or_sphere *solids, int nsolids, const or_sim *s) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  const double dRho = s->rhoL - s->rhoG;
  for (int z = 1; z < nz - 1; z++)
    for (int y = 1; y < ny - 1; y++)
      for (int x = 1; x < nx - 1; x++) {
        int i = ((z * ny) + y) * nx + x;
        if (s->tag[i] != 1 || s->tagPrev[i] != 0) continue;
        double rhoPhase = s->rhoG + (double)s->phi[i] * dRho;
        int b = owner_of(solids, nsolids, x, y, z);
        if (b < 0) continue;
        or_sphere_apply_impulse(&solids[b], x, y, z, rhoPhase * (double)s->ux[i],
                                rhoPhase * (double)s->uy[i], rhoPhase * (double)s->uz[i]);
      }
}

/* Math.max / Math.min semantics for the wall clamp (NaN propagates, +0 > -0). */
static double js_max0(double v) {
  if (v != v) return v;
  if (v == 0) return signbit(v) ? 0.0 : v;
  return v > 0 ? v : 0.0;
}
static double js_min0(double v) {
  if (v != v) return v;
  if (v == 0) return signbit(v) ? v : 0.0;
  return v < 0 ? v : 0.0;
}

/* src/solid.js:104-210 */
void or_sphere_step(or_sphere *b, double dt, double gravity) {
  double bodyG = gravity;
  b->Fy += b->mass * bodyG;
  if (b->dragging) {
    double k = 0.004 * b->mass;
    double cD = 2.0 * sqrt(k * b->mass);
    b->Fx += k * (b->dragTargetX - b->cx) - cD * b->vx;
    b->Fy += k * (b->dragTargetY - b->cy) - cD * b->vy;
    b->Fz += k * (b->dragTargetZ - b->cz) - cD * b->vz;
  }
  /* `gravity || 0.001`: 0, -0 and NaN are falsy */
  double gsel = (gravity == 0 || gravity != gravity) ? 0.001 : gravity;
  double accCap = 3.5 * fabs(gsel);
  {
    double ax = b->Fx / b->mass;
    double ay = b->Fy / b->mass;
    double az = b->Fz / b->mass;
    double a2 = ax * ax + ay * ay + az * az;
    double c2 = accCap * accCap;
    double sc = a2 > c2 ? accCap / sqrt(a2) : 1.0;
    b->vx += dt * ax * sc;
    b->vy += dt * ay * sc;
    b->vz += dt * az * sc;
  }
  b->wx += dt * b->Tx / b->I;
  b->wy += dt * b->Ty / b->I;
  b->wz += dt * b->Tz / b->I;
  const double BODY_UMAX = 0.08;
  double sp2 = b->vx * b->vx + b->vy * b->vy + b->vz * b->vz;
  if (sp2 > BODY_UMAX * BODY_UMAX) {
    double sc = BODY_UMAX / sqrt(sp2);
    b->vx *= sc;
    b->vy *= sc;
    b->vz *= sc;
  }
  const double linDamp = 0.98, omegaDamp = 0.95;
  b->vx *= linDamp;
  b->vy *= linDamp;
  b->vz *= linDamp;
  b->wx *= omegaDamp;
  b->wy *= omegaDamp;
  b->wz *= omegaDamp;
  const double SNAP = 0.0001;
  if (fabs(b->vx) < SNAP) b->vx = 0;
  if (fabs(b->vy) < SNAP) b->vy = 0;
  if (fabs(b->vz) < SNAP) b->vz = 0;
  if (fabs(b->wx) < SNAP) b->wx = 0;
  if (fabs(b->wy) < SNAP) b->wy = 0;
  if (fabs(b->wz) < SNAP) b->wz = 0;
  b->cx += dt * b->vx;
  b->cy += dt * b->vy;
  b->cz += dt * b->vz;
  double m = b->r + 1.5;
  if (b->cx < m) { b->cx = m; b->vx = js_max0(b->vx); }
  if (b->cx > b->nx - 1 - m) { b->cx = b->nx - 1 - m; b->vx = js_min0(b->vx); }
  if (b->cy < m) { b->cy = m; b->vy = js_max0(b->vy); }
  if (b->cy > b->ny - 1 - m) { b->cy = b->ny - 1 - m; b->vy = js_min0(b->vy); }
  if (b->cz < m) { b->cz = m; b->vz = js_max0(b->vz); }
  if (b->cz > b->nz - 1 - m) { b->cz = b->nz - 1 - m; b->vz = js_min0(b->vz); }
  b->Fx = b->Fy = b->Fz = 0;
  b->Tx = b->Ty = b->Tz = 0;
}

/* src/worker.js:96-100 */
void or_worker_substep(or_sim *s, or_sphere *solids, int nsolids) {
  or_step(s, solids, nsolids);
  if (solids && nsolids > 0) {
    or_absorb_dead_cells(solids, nsolids, s);
    for (int b = 0; b < nsolids; b++) or_sphere_step(&solids[b], 1.0, s->gravity);
  }
}
