/*
 * ws_oracle.c — TEST INFRASTRUCTURE ONLY: CPU restatement of WaterSim's
 * FluidSolver (js/solver.js) for parity checks of the CUDA library.
 * Never linked into the product; see ws_oracle.h.
 *
 * JS semantics are kept literally: storage arrays have type st_t (float for
 * the js build: every store into a Float32Array rounds to float32), every
 * local is a double (JS numbers), `|0` truncates toward zero, `>>> 0`
 * reduces mod 2^32. Build with -ffp-contract=off so no multiply-add is fused
 * (JS never fuses). Each function cites the solver.js lines it restates.
 */
#include "ws_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>

#ifndef OR_ST
#define OR_ST float
#endif
typedef OR_ST st_t;

enum { AIR = 0, FLUID = 1, SOLID = 2 };
#define OR_MAX_BALLS 64
enum { BX, BY, BZ, BVX, BVY, BVZ, BR, BRHO, BSUB };
#define EVAP_STEEPNESS 3.5               /* js/solver.js:40 */

struct or_solver {
  int nx, ny, nz; double dx;
  double W, H, D, cx, cy, cz, domainR;
  int nCells, uN, vN, wN;
  or_params P;
  or_scalars S;
  uint8_t *cellType; st_t *cellPhi, *svx, *svy, *svz;
  st_t *u, *v, *w, *uW, *vW, *wW, *uO, *vO, *wO;
  uint8_t *validU, *validV, *validW;
  int32_t *nb; st_t *diag, *rhs, *q;
  st_t *dens;
  st_t *px, *py, *pz, *pvx, *pvy, *pvz, *pT, *pAir, *pLight, *pWx, *pWy, *pWz, *pPh;
  uint8_t *pflag, *pcool, *pDepth;
  double *advU, *advV, *advW;
  int hasTerr; int tn; double tdv; uint8_t *tsolid; st_t *tR;
  double Rsl, Rlo, Rhi, Rlo2, Rhi2;
  uint8_t *staticTypes; int staticValid;
  st_t *gu, *gv, *gw; int hasGravity;
  int32_t *fluidList; int nFluid;
  st_t *vcx, *vcy, *vcz, *omg, *omx, *omy, *omz;
  int32_t *steamCnt;
  int32_t *hCnt, *hStart, *hCur, *hOrd; int hOrdCap;
  double *heatMean, *heatDelta; double heatDt, heatAlpha;
  int32_t *pStart, *pAdj; st_t *pW; int pCap;
  int32_t *vIdx, *iceIdx; int idxCap;
  int gridSampleValid;
  /* balls (addBall, js/solver.js:3910-3912): x y z vx vy vz r rho submerged */
  double balls[OR_MAX_BALLS][9]; int nBalls; int hadSolidVelocity;
  float surfY[OR_MAX_BALLS];
};

/* ------------------------------------------------------------ helpers */
static inline double jclampd(double v, double a, double b) { return v < a ? a : (v > b ? b : v); }
static inline int jfloor_clamp(double v, int a, int b) {     /* clamp(Math.floor(v), a, b) */
  double f = floor(v);
  if (f < a) return a;
  if (f > b) return b;
  return (int)f;
}
static inline int jtrunc(double v) { return (int)v; }        /* v | 0 for |v| < 2^31 */
static inline int jceil_clamp(double v, int a, int b) {      /* clamp(Math.ceil(v), a, b) */
  double f = ceil(v);
  if (f < a) return a;
  if (f > b) return b;
  return (int)f;
}
static inline uint32_t lcg(uint32_t s) { return s * 1664525u + 1013904223u; }
static inline double jmin(double a, double b) { return a < b ? a : b; }
static inline double jmax(double a, double b) { return a > b ? a : b; }
static void* xcalloc(size_t n, size_t sz) { void* p = calloc(n ? n : 1, sz); return p; }

int or_storage_bytes(void) { return (int)sizeof(st_t); }

/* ------------------------------------------------------------ construction
 * js/solver.js:45-216 (sphere mode). */
or_solver* or_create(int nx, int ny, int nz, double dx, double coreR,
                     uint32_t terrainSeed, double bumpiness, double targetParticles) {
  or_solver* s = (or_solver*)xcalloc(1, sizeof(or_solver));
  s->nx = nx; s->ny = ny; s->nz = nz; s->dx = dx;
  s->W = nx * dx; s->H = ny * dx; s->D = nz * dx;
  s->cx = s->W / 2; s->cy = s->H / 2; s->cz = s->D / 2;
  s->domainR = 0.5 * jmin(jmin(s->W, s->H), s->D) - dx;
  s->nCells = nx * ny * nz;
  s->uN = (nx + 1) * ny * nz; s->vN = nx * (ny + 1) * nz; s->wN = nx * ny * (nz + 1);
  int N = s->nCells;
  s->cellType = xcalloc(N, 1);
  s->svx = xcalloc(N, sizeof(st_t)); s->svy = xcalloc(N, sizeof(st_t)); s->svz = xcalloc(N, sizeof(st_t));
  s->cellPhi = xcalloc(N, sizeof(st_t));
  s->u = xcalloc(s->uN, sizeof(st_t)); s->v = xcalloc(s->vN, sizeof(st_t)); s->w = xcalloc(s->wN, sizeof(st_t));
  s->uW = xcalloc(s->uN, sizeof(st_t)); s->vW = xcalloc(s->vN, sizeof(st_t)); s->wW = xcalloc(s->wN, sizeof(st_t));
  s->uO = xcalloc(s->uN, sizeof(st_t)); s->vO = xcalloc(s->vN, sizeof(st_t)); s->wO = xcalloc(s->wN, sizeof(st_t));
  s->validU = xcalloc(s->uN, 1); s->validV = xcalloc(s->vN, 1); s->validW = xcalloc(s->wN, 1);
  s->nb = xcalloc((size_t)N * 6, sizeof(int32_t));
  s->diag = xcalloc(N, sizeof(st_t)); s->rhs = xcalloc(N, sizeof(st_t)); s->q = xcalloc(N, sizeof(st_t));
  s->dens = xcalloc((size_t)(nx + 1) * (ny + 1) * (nz + 1), sizeof(st_t));
  s->staticTypes = xcalloc(N, 1);
  s->fluidList = xcalloc(N, sizeof(int32_t));
  s->steamCnt = xcalloc(N, sizeof(int32_t));
  s->vcx = xcalloc(N, sizeof(st_t)); s->vcy = xcalloc(N, sizeof(st_t)); s->vcz = xcalloc(N, sizeof(st_t));
  s->omg = xcalloc(N, sizeof(st_t)); s->omx = xcalloc(N, sizeof(st_t));
  s->omy = xcalloc(N, sizeof(st_t)); s->omz = xcalloc(N, sizeof(st_t));
  s->hCnt = xcalloc(N, sizeof(int32_t)); s->hStart = xcalloc(N + 1, sizeof(int32_t));
  s->hCur = xcalloc(N, sizeof(int32_t));
  s->heatMean = xcalloc(N, sizeof(double)); s->heatDelta = xcalloc(N, sizeof(double));
  /* knobs: library defaults (js/solver.js:56-193) */
  or_params* P = &s->P;
  P->substeps = 1; P->cfl = 3.0; P->pic = 0.15; P->gravity = 9.81; P->viscosity = 5e-4;
  P->pressureIters = 20; P->omega = 1.55; P->maxSpeed = 3.2;
  P->vorticity = 0; P->currents = 0; P->shadeCool = 0.035;
  P->sunActivity = 0; P->evapIntensity = 0.05; P->atmosphereH = 0.35; P->ceilReflect = 0;
  P->hasSun = 0; P->heatK = 0.6; P->Tamb = 0.32;
  P->cloudT = 0.34; P->cloudP = 0.35; P->rainT = 0.22; P->rainLiftAge = 0.4; P->snowT = 0.10;
  P->meltT = P->snowT * 1.05; P->spinOn = 0; P->thermalOn = 1;
  P->sorRedBlack = 0; P->sorCheckEvery = 10; P->sorTol = 0; P->sorMaxIters = 10000;
  P->viscJacobi = 0; P->extrapJacobi = 0;
  or_scalars* S = &s->S;
  S->coreR = coreR; S->oceanR = 0; S->spacing = dx * 0.5;
  S->particleVolume = S->spacing * S->spacing * S->spacing; S->iso = 1.8; S->waterTopY = dx + 1;
  S->gRamp = 1e9; S->evS = 0x51ab3c77u; S->cfS = 0x2f6e2b1u; S->bfS = 0x7f4a7c15u;
  S->stirS = 0x2545f491u;
  S->terrainSeed = terrainSeed ? terrainSeed : 20260114u;
  S->bumpiness = bumpiness < 0 ? 0 : (bumpiness > 2.5 ? 2.5 : bumpiness);
  S->targetParticles = targetParticles > 0 ? targetParticles : 110000;
  or_alloc_particles(s, 1);
  s->S.capacity = 1;
  return s;
}

static void free_particles(or_solver* s) {
  free(s->px); free(s->py); free(s->pz); free(s->pvx); free(s->pvy); free(s->pvz);
  free(s->pflag); free(s->pcool); free(s->pT); free(s->pAir); free(s->pLight); free(s->pDepth);
  free(s->pWx); free(s->pWy); free(s->pWz); free(s->pPh);
  free(s->advU); free(s->advV); free(s->advW);
}

/* js/solver.js:218-231 (arrays are re-created zeroed, as the JS allocator does) */
int or_alloc_particles(or_solver* s, int cap) {
  if (s->S.capacity >= cap && s->px) return 0;
  free_particles(s);
  s->S.capacity = cap;
  s->px = xcalloc(cap, sizeof(st_t)); s->py = xcalloc(cap, sizeof(st_t)); s->pz = xcalloc(cap, sizeof(st_t));
  s->pvx = xcalloc(cap, sizeof(st_t)); s->pvy = xcalloc(cap, sizeof(st_t)); s->pvz = xcalloc(cap, sizeof(st_t));
  s->pflag = xcalloc(cap, 1); s->pcool = xcalloc(cap, 1);
  s->pT = xcalloc(cap, sizeof(st_t)); s->pAir = xcalloc(cap, sizeof(st_t)); s->pLight = xcalloc(cap, sizeof(st_t));
  s->pDepth = xcalloc(cap, 1);
  s->pWx = xcalloc(cap, sizeof(st_t)); s->pWy = xcalloc(cap, sizeof(st_t)); s->pWz = xcalloc(cap, sizeof(st_t));
  s->pPh = xcalloc(cap, sizeof(st_t));
  s->advU = xcalloc(cap, sizeof(double)); s->advV = xcalloc(cap, sizeof(double)); s->advW = xcalloc(cap, sizeof(double));
  return 0;
}

void or_destroy(or_solver* s) {
  if (!s) return;
  free_particles(s);
  free(s->cellType); free(s->svx); free(s->svy); free(s->svz); free(s->cellPhi);
  free(s->u); free(s->v); free(s->w); free(s->uW); free(s->vW); free(s->wW);
  free(s->uO); free(s->vO); free(s->wO); free(s->validU); free(s->validV); free(s->validW);
  free(s->nb); free(s->diag); free(s->rhs); free(s->q); free(s->dens); free(s->staticTypes);
  free(s->fluidList); free(s->steamCnt);
  free(s->vcx); free(s->vcy); free(s->vcz); free(s->omg); free(s->omx); free(s->omy); free(s->omz);
  free(s->hCnt); free(s->hStart); free(s->hCur); free(s->hOrd); free(s->heatMean); free(s->heatDelta);
  free(s->pStart); free(s->pAdj); free(s->pW); free(s->vIdx); free(s->iceIdx);
  free(s->tsolid); free(s->tR); free(s->gu); free(s->gv); free(s->gw);
  free(s);
}

void or_get_params(const or_solver* s, or_params* p) { *p = s->P; }
void or_set_params(or_solver* s, const or_params* p) { s->P = *p; }
void or_get_scalars(const or_solver* s, or_scalars* o) { *o = s->S; o->nFluid = s->nFluid; }
void or_set_scalars(or_solver* s, const or_scalars* o) {
  int cap = s->S.capacity;
  s->S = *o;
  s->S.capacity = cap;
  s->nFluid = o->nFluid;
}

void* or_array(or_solver* s, const char* nm, int64_t* count, int* kind) {
  int64_t N = s->nCells, P = s->S.capacity;
  int64_t T = s->hasTerr ? (int64_t)s->tn * s->tn * s->tn : 0;
#define A(name_, ptr_, cnt_, kind_) if (!strcmp(nm, name_)) { *count = (cnt_); *kind = (kind_); return (void*)(ptr_); }
  A("cellType", s->cellType, N, 0) A("staticTypes", s->staticTypes, N, 0)
  A("q", s->q, N, 2) A("rhs", s->rhs, N, 2) A("diag", s->diag, N, 2) A("cellPhi", s->cellPhi, N, 2)
  A("u", s->u, s->uN, 2) A("v", s->v, s->vN, 2) A("w", s->w, s->wN, 2)
  A("uW", s->uW, s->uN, 2) A("vW", s->vW, s->vN, 2) A("wW", s->wW, s->wN, 2)
  A("uO", s->uO, s->uN, 2) A("vO", s->vO, s->vN, 2) A("wO", s->wO, s->wN, 2)
  A("validU", s->validU, s->uN, 0) A("validV", s->validV, s->vN, 0) A("validW", s->validW, s->wN, 0)
  A("dens", s->dens, (int64_t)(s->nx + 1) * (s->ny + 1) * (s->nz + 1), 2)
  A("px", s->px, P, 2) A("py", s->py, P, 2) A("pz", s->pz, P, 2)
  A("pvx", s->pvx, P, 2) A("pvy", s->pvy, P, 2) A("pvz", s->pvz, P, 2)
  A("pT", s->pT, P, 2) A("pAir", s->pAir, P, 2) A("pLight", s->pLight, P, 2)
  A("pWx", s->pWx, P, 2) A("pWy", s->pWy, P, 2) A("pWz", s->pWz, P, 2) A("pPh", s->pPh, P, 2)
  A("pflag", s->pflag, P, 0) A("pcool", s->pcool, P, 0) A("pDepth", s->pDepth, P, 0)
  A("advU", s->advU, P, 3) A("advV", s->advV, P, 3) A("advW", s->advW, P, 3)
  A("tsolid", s->tsolid, T, 0) A("tR", s->tR, T, 2)
  A("gu", s->gu, s->hasGravity ? s->uN : 0, 2) A("gv", s->gv, s->hasGravity ? s->vN : 0, 2)
  A("gw", s->gw, s->hasGravity ? s->wN : 0, 2)
  A("fluidList", s->fluidList, s->nFluid, 1)
#undef A
  *count = 0; *kind = -1;
  return NULL;
}

/* ------------------------------------------------------------ terrain
 * Seeded value noise, js/solver.js:236-262. */
typedef struct { uint8_t perm[512]; } tnoise;
static void tnoise_init(tnoise* t, uint32_t seed) {
  uint8_t base[256]; uint32_t s = seed; int i, j;
  for (i = 0; i < 256; i++) base[i] = (uint8_t)i;
  for (i = 255; i > 0; i--) {
    s = lcg(s);
    j = (int)((s >> 8) % (uint32_t)(i + 1));
    uint8_t t0 = base[i]; base[i] = base[j]; base[j] = t0;
  }
  for (i = 0; i < 512; i++) t->perm[i] = base[i & 255];
}
static inline double tn_h(const tnoise* t, int ix, int iy, int iz) {
  return t->perm[(t->perm[(t->perm[ix & 255] + iy) & 255] + iz) & 255] / 255.0;
}
static inline double tn_fade(double u) { return u * u * u * (u * (u * 6 - 15) + 10); }
static double tn_eval(const tnoise* t, double x, double y, double z) {
  double fx = floor(x), fy = floor(y), fz = floor(z);
  int ix = (int)fx, iy = (int)fy, iz = (int)fz;
  double u = tn_fade(x - fx), v = tn_fade(y - fy), w = tn_fade(z - fz);
  double a = tn_h(t, ix, iy, iz), b = tn_h(t, ix + 1, iy, iz);
  double c = tn_h(t, ix, iy + 1, iz), d = tn_h(t, ix + 1, iy + 1, iz);
  double e = tn_h(t, ix, iy, iz + 1), f = tn_h(t, ix + 1, iy, iz + 1);
  double g = tn_h(t, ix, iy + 1, iz + 1), hh = tn_h(t, ix + 1, iy + 1, iz + 1);
  double x1 = a + (b - a) * u, x2 = c + (d - c) * u;
  double x3 = e + (f - e) * u, x4 = g + (hh - g) * u;
  double y1 = x1 + (x2 - x1) * v, y2 = x3 + (x4 - x3) * v;
  return y1 + (y2 - y1) * w;
}
/* rawHeight, js/solver.js:292-313 */
static double raw_height(const tnoise* nf, double bump, double dx, double dy, double dz) {
  double wx = tn_eval(nf, dx * 0.9 + 17.3, dy * 0.9 + 9.1, dz * 0.9 + 4.7) - 0.5;
  double wy = tn_eval(nf, dx * 0.9 + 71.9, dy * 0.9 + 33.7, dz * 0.9 + 21.3) - 0.5;
  double wz = tn_eval(nf, dx * 0.9 + 123.4, dy * 0.9 + 87.2, dz * 0.9 + 55.8) - 0.5;
  double qx = dx + 0.35 * wx, qy = dy + 0.35 * wy, qz = dz + 0.35 * wz;
  double h = 0, amp = 1, fr = 1.15, tot = 0, v; int o;
  for (o = 0; o < 4; o++) {
    h += amp * tn_eval(nf, qx * fr + 3.1, qy * fr + 7.7, qz * fr + 11.9);
    tot += amp; amp *= 0.5; fr *= 2.1;
  }
  h /= tot;
  double r = 0; amp = 1; fr = 2.6; tot = 0;
  for (o = 0; o < 3; o++) {
    v = tn_eval(nf, qx * fr + 41.2, qy * fr + 23.8, qz * fr + 66.1);
    r += amp * (1 - fabs(2 * v - 1));
    tot += amp; amp *= 0.55; fr *= 2.3;
  }
  r /= tot;
  double det = tn_eval(nf, qx * 6.5 + 91.7, qy * 6.5 + 12.4, qz * 6.5 + 78.3);
  return h + 0.45 * bump * (r - 0.5) + 0.14 * bump * (det - 0.5);
}

/* generateTerrain, js/solver.js:272-508. The renderer's corner field
 * (:433-481) is display-only and not built. */
void or_generate_terrain(or_solver* s, uint32_t seed, double seaLevel) {
  double R1 = s->S.coreR, Rsl = seaLevel, bump = s->S.bumpiness;
  double depthW = jmax(Rsl - R1, 1e-4);
  double Rlo = jmax(R1 * 0.55, Rsl - 1.8889 * depthW);
  double Rhi = Rsl + 0.7778 * depthW;
  double span = Rhi - Rlo;
  double mW = jmin(1, bump / 0.3);
  double Rsph = Rsl - jmin(0.4 * depthW, 0.45 * (Rsl - Rlo));
  tnoise nf; tnoise_init(&nf, seed);
  enum { CALN = 8192 };
  float* cal = (float*)malloc(sizeof(float) * CALN);      /* Float32Array in JS */
  uint32_t cs = seed;
#define CRND() (cs = lcg(cs), cs / 4294967296.0)
  double cMin = 1e9, cMax = -1e9; int ci;
  for (ci = 0; ci < CALN; ci++) {
    double u1 = CRND() * 2 - 1; double th = CRND() * 6.2831853;
    double sq = sqrt(1 - u1 * u1);
    double hv = raw_height(&nf, bump, sq * cos(th), u1, sq * sin(th));
    cal[ci] = (float)hv;
    if (hv < cMin) cMin = hv; else if (hv > cMax) cMax = hv;
  }
  double cSpan = (cMax - cMin); if (cSpan == 0) cSpan = 1;
  double hSl = (Rsl - Rlo) / span;
  double lo = -1, hi = 1, delta = 0; int it, cnt;
  for (it = 0; it < 48; it++) {
    delta = 0.5 * (lo + hi);
    cnt = 0;
    for (ci = 0; ci < CALN; ci++) {
      double h01 = (cal[ci] - cMin) / cSpan;
      double hs = h01 + delta; if (hs < 0) hs = 0; else if (hs > 1) hs = 1;
      if (pow(hs, 1.25) > hSl) cnt++;
    }
    if (cnt > 0.27 * CALN) hi = delta; else lo = delta;
  }
  double offs = delta;
  free(cal);
  double dv = s->dx / 2;
  int n = (int)ceil(s->W / dv);
  size_t n3 = (size_t)n * n * n;
  free(s->tsolid); free(s->tR);
  uint8_t* solid = (uint8_t*)xcalloc(n3, 1);
  st_t* R = (st_t*)xcalloc(n3, sizeof(st_t));
  double cx = s->cx, cy = s->cy, cz = s->cz;
  int iv, jv, kv; size_t idx;
  for (kv = 0; kv < n; kv++) {
    double pz0 = (kv + 0.5) * dv - cz;
    for (jv = 0; jv < n; jv++) {
      double py0 = (jv + 0.5) * dv - cy;
      for (iv = 0; iv < n; iv++) {
        double px0 = (iv + 0.5) * dv - cx;
        double rr = sqrt(px0 * px0 + py0 * py0 + pz0 * pz0);
        idx = ((size_t)kv * n + jv) * n + iv;
        if (rr < 1e-6) { R[idx] = (st_t)Rlo; solid[idx] = 1; continue; }
        double rv;
        if (mW <= 0) rv = Rsph;
        else {
          double hv = raw_height(&nf, bump, px0 / rr, py0 / rr, pz0 / rr);
          double h01 = (hv - cMin) / cSpan + offs;
          if (h01 < 0) h01 = 0; else if (h01 > 1) h01 = 1;
          double rvv = Rlo + pow(h01, 1.25) * span;
          rv = Rsph + (rvv - Rsph) * mW;
        }
        R[idx] = (st_t)rv;
        if (rr <= rv) solid[idx] = 1;
      }
    }
  }
  /* slope smoothing, js/solver.js:384-426 (in place, fixed order) */
  int PASSES = n < 48 ? 1 : (n < 64 ? 2 : 3);
  double BLEND = n < 48 ? 0.15 : (n < 64 ? 0.35 : 0.5);
  long sN = n, sN2 = (long)n * n; int ps;
  for (ps = 0; ps < PASSES; ps++) {
    for (kv = 1; kv < sN - 1; kv++) {
      long zBase = kv * sN2, zBaseL = (kv - 1) * sN2, zBaseU = (kv + 1) * sN2;
      for (jv = 1; jv < sN - 1; jv++) {
        long yBase = zBase + jv * sN, yBaseL = zBaseL + (jv - 1) * sN, yBaseU = zBaseL + (jv + 1) * sN;
        long yBase2 = zBaseU + (jv - 1) * sN, yBase3 = zBaseU + jv * sN, yBase4 = zBaseU + (jv + 1) * sN;
        long yBaseL2 = zBase + (jv - 1) * sN, yBaseU2 = zBase + (jv + 1) * sN;
        for (iv = 1; iv < sN - 1; iv++) {
          long iR = yBase + iv;
          double avg = ((double)R[iR - 1] + R[iR + 1] + R[yBaseL2 + iv] + R[yBaseU2 + iv] +
                        R[yBaseL + iv] + R[yBase2 + iv] + R[yBase3 + iv] + R[yBase4 + iv] +
                        R[yBaseL + iv - 1] + R[yBaseL + iv + 1] + R[yBase2 + iv - 1] + R[yBase2 + iv + 1] +
                        R[yBaseU + iv] + R[yBase3 + iv - 1] + R[yBase3 + iv + 1] + R[yBase4 + iv] +
                        R[yBaseL2 + iv - 1] + R[yBaseL2 + iv + 1]) * (1.0 / 18);
          R[iR] = (st_t)(R[iR] + (avg - R[iR]) * BLEND);
        }
      }
    }
  }
  double mean0 = 0, mean1 = 0; long cntR = 0;
  for (idx = 0; idx < n3; idx += 7) { mean0 += R[idx]; cntR++; }
  mean0 /= cntR;
  for (ps = 0; ps < PASSES; ps++) {
    for (kv = 1; kv < sN - 1; kv++) for (jv = 1; jv < sN - 1; jv++) {
      long rowS = kv * sN2 + jv * sN;
      for (iv = 1; iv < sN - 1; iv++) {
        long iS = rowS + iv;
        double avg2 = ((double)R[iS - 1] + R[iS + 1] + R[iS - sN] + R[iS + sN] +
                       R[iS - sN2] + R[iS + sN2]) * (1.0 / 6);
        R[iS] = (st_t)(R[iS] + (avg2 - R[iS]) * BLEND);
      }
    }
  }
  for (idx = 0; idx < n3; idx += 7) mean1 += R[idx];
  mean1 /= cntR;
  if (mean1 > 1e-9) {
    double rScale = mean0 / mean1;
    for (idx = 0; idx < n3; idx++) R[idx] = (st_t)(R[idx] * rScale);
  }
  for (kv = 0; kv < n; kv++) {
    double pzS = (kv + 0.5) * dv - cz;
    for (jv = 0; jv < n; jv++) {
      double pyS = (jv + 0.5) * dv - cy;
      size_t rowS2 = ((size_t)kv * n + jv) * n;
      for (iv = 0; iv < n; iv++) {
        double pxS = (iv + 0.5) * dv - cx;
        double rrS = sqrt(pxS * pxS + pyS * pyS + pzS * pzS);
        idx = rowS2 + iv;
        solid[idx] = rrS <= R[idx] ? 1 : 0;
      }
    }
  }
  /* land fraction on the voxels, js/solver.js:484-497 */
  int LANDN = 4000, land = 0;
  for (ci = 0; ci < LANDN; ci++) {
    double lu = CRND() * 2 - 1; double lth = CRND() * 6.2831853;
    double lsq = sqrt(1 - lu * lu);
    double ldx = lsq * cos(lth), ldy = lu, ldz = lsq * sin(lth);
    double rr2;
    for (rr2 = Rhi + dv; rr2 > Rlo - dv; rr2 -= dv * 0.5) {
      int sx = jtrunc((cx + ldx * rr2) / dv), sy = jtrunc((cy + ldy * rr2) / dv), sz = jtrunc((cz + ldz * rr2) / dv);
      if (sx < 0 || sy < 0 || sz < 0 || sx >= n || sy >= n || sz >= n) continue;
      if (solid[((size_t)sz * n + sy) * n + sx]) {
        if (rr2 > Rsl) land++;
        break;
      }
    }
  }
#undef CRND
  s->hasTerr = 1; s->tn = n; s->tdv = dv; s->tsolid = solid; s->tR = R;
  s->Rsl = Rsl; s->Rlo = Rlo; s->Rhi = Rhi; s->Rlo2 = Rlo * Rlo; s->Rhi2 = Rhi * Rhi;
  s->S.landFrac = (double)land / LANDN;
  s->staticValid = 0;
}

int or_load_terrain(or_solver* s, int n, double dv, const uint8_t* solid, const void* R,
                    double Rsl, double Rlo, double Rhi, double landFrac) {
  size_t n3 = (size_t)n * n * n;
  free(s->tsolid); free(s->tR);
  s->tsolid = (uint8_t*)malloc(n3); memcpy(s->tsolid, solid, n3);
  s->tR = (st_t*)malloc(n3 * sizeof(st_t));
  const float* Rf = (const float*)R;          /* terrain fixtures are float32 */
  for (size_t i = 0; i < n3; i++) s->tR[i] = (st_t)Rf[i];
  s->hasTerr = 1; s->tn = n; s->tdv = dv;
  s->Rsl = Rsl; s->Rlo = Rlo; s->Rhi = Rhi; s->Rlo2 = Rlo * Rlo; s->Rhi2 = Rhi * Rhi;
  s->S.landFrac = landFrac;
  s->staticValid = 0;
  return 0;
}

/* terrainRadiusAt, js/solver.js:512-535 */
double or_terrain_radius_at(or_solver* s, double x, double y, double z) {
  if (!s->hasTerr) return s->S.coreR;
  int n = s->tn; double dv = s->tdv; const st_t* R = s->tR;
  double gx = x / dv - 0.5, gy = y / dv - 0.5, gz = z / dv - 0.5;
  int i = jtrunc(gx), j = jtrunc(gy), k = jtrunc(gz);
  if (i < 0) i = 0; else if (i > n - 2) i = n - 2;
  if (j < 0) j = 0; else if (j > n - 2) j = n - 2;
  if (k < 0) k = 0; else if (k > n - 2) k = n - 2;
  double fx = gx - i, fy = gy - j, fz = gz - k;
  if (fx < 0) fx = 0; else if (fx > 1) fx = 1;
  if (fy < 0) fy = 0; else if (fy > 1) fy = 1;
  if (fz < 0) fz = 0; else if (fz > 1) fz = 1;
  size_t b000 = ((size_t)k * n + j) * n + i, s7 = (size_t)n * n;
  double v000 = R[b000], v100 = R[b000 + 1];
  double v010 = R[b000 + n], v110 = R[b000 + n + 1];
  double v001 = R[b000 + s7], v101 = R[b000 + s7 + 1];
  double v011 = R[b000 + s7 + n], v111 = R[b000 + s7 + n + 1];
  double a0 = v000 + (v100 - v000) * fx, a1 = v010 + (v110 - v010) * fx;
  double a2 = v001 + (v101 - v001) * fx, a3 = v011 + (v111 - v011) * fx;
  double b0 = a0 + (a1 - a0) * fy, b1 = a2 + (a3 - a2) * fy;
  return b0 + (b1 - b0) * fz;
}

/* _rockCellAt, js/solver.js:542-559 (the cached-static-types path and the
 * voxel path agree for the clamped indices, so the voxel rule is used). */
int or_rock_cell_at(or_solver* s, double x, double y, double z) {
  if (!s->hasTerr) return 0;
  double dx = s->dx; int nx = s->nx, ny = s->ny, nz = s->nz;
  int i = jtrunc(x / dx), j = jtrunc(y / dx), k = jtrunc(z / dx);
  if (i < 1) i = 1; else if (i > nx - 2) i = nx - 2;
  if (j < 1) j = 1; else if (j > ny - 2) j = ny - 2;
  if (k < 1) k = 1; else if (k > nz - 2) k = nz - 2;
  int tvn = s->tn; double tvd = s->tdv;
  int vx = jtrunc((i + 0.5) * dx / tvd), vy = jtrunc((j + 0.5) * dx / tvd), vz = jtrunc((k + 0.5) * dx / tvd);
  if (vx < 0) vx = 0; else if (vx >= tvn) vx = tvn - 1;
  if (vy < 0) vy = 0; else if (vy >= tvn) vy = tvn - 1;
  if (vz < 0) vz = 0; else if (vz >= tvn) vz = tvn - 1;
  return s->tsolid[((size_t)vz * tvn + vy) * tvn + vx] == 1;
}
#define ROCK(s_, x_, y_, z_) or_rock_cell_at((s_), (x_), (y_), (z_))
#define TRAD(s_, x_, y_, z_) or_terrain_radius_at((s_), (x_), (y_), (z_))

/* _voxelRockAt, js/solver.js:565-574 */
static int voxel_rock_at(or_solver* s, double x, double y, double z) {
  if (!s->hasTerr) return 0;
  int n = s->tn; double dv = s->tdv;
  int i = jtrunc(x / dv), j = jtrunc(y / dv), k = jtrunc(z / dv);
  if (i < 0) i = 0; else if (i > n - 1) i = n - 1;
  if (j < 0) j = 0; else if (j > n - 1) j = n - 1;
  if (k < 0) k = 0; else if (k > n - 1) k = n - 1;
  return s->tsolid[((size_t)k * n + j) * n + i] == 1;
}

/* _onRockBelow, js/solver.js:581-587 */
static int on_rock_below(or_solver* s, double x, double y, double z) {
  if (!s->hasTerr) return 0;
  double ex = x - s->cx, ey = y - s->cy, ez = z - s->cz;
  double el = sqrt(ex * ex + ey * ey + ez * ez); if (el == 0) el = 1e-9;
  double sc = s->dx * 0.9 / el;
  return ROCK(s, x - ex * sc, y - ey * sc, z - ez * sc);
}

/* ------------------------------------------------------------ water fill
 * Monte-Carlo water volume, js/solver.js:661-675. */
double or_water_volume_mc(or_solver* s, double depth) {
  double R1 = s->S.coreR, R2 = R1 + depth;
  uint32_t seed = s->S.terrainSeed;
  double Rlo = s->Rlo;
  double Vshell = 4.0 / 3 * M_PI * (R2 * R2 * R2 - Rlo * Rlo * Rlo);
  int MC = 20000, hits = 0, mi; uint32_t mcS = seed ^ 0x9e3779b9u;
  double cx = s->cx, cy = s->cy, cz = s->cz;
  for (mi = 0; mi < MC; mi++) {
    mcS = lcg(mcS); double u1 = mcS / 4294967296.0 * 2 - 1;
    mcS = lcg(mcS); double th = mcS / 4294967296.0 * 6.2831853;
    double sq = sqrt(1 - u1 * u1);
    mcS = lcg(mcS);
    double rr = cbrt(Rlo * Rlo * Rlo + mcS / 4294967296.0 * (R2 * R2 * R2 - Rlo * Rlo * Rlo));
    double qx = cx + sq * cos(th) * rr, qy = cy + u1 * rr, qz = cz + sq * sin(th) * rr;
    if (!ROCK(s, qx, qy, qz)) hits++;
  }
  return Vshell * hits / MC;
}

/* _resetWaterSphere, js/solver.js:651-731 (the terrain must already exist
 * for (coreR, coreR+depth); or_generate_terrain is the generator). */
void or_reset_water(or_solver* s, double depth) {
  s->nBalls = 0;
  double R1 = s->S.coreR, R2 = R1 + depth;
  s->S.oceanR = R2;
  uint32_t seed = s->S.terrainSeed;
  if (!s->hasTerr) or_generate_terrain(s, seed, R2);
  double Vw = or_water_volume_mc(s, depth);
  double sp = cbrt(Vw / s->S.targetParticles);
  s->S.spacing = sp;
  s->S.particleVolume = sp * sp * sp;
  double rHi = R2 - 0.4 * sp;
  int cap = (int)(s->S.targetParticles + 8192);
  or_alloc_particles(s, cap);
  double cx = s->cx, cy = s->cy, cz = s->cz;
  uint32_t fjS = seed ^ 0x51ab3c77u;
  int n = 0; double x, y, z;
  for (y = cy - R2; y <= cy + R2; y += sp) {
    for (z = cz - R2; z <= cz + R2; z += sp) {
      for (x = cx - R2; x <= cx + R2; x += sp) {
        if (n >= cap) break;
        double ex = x - cx, ey = y - cy, ez = z - cz;
        double r2 = ex * ex + ey * ey + ez * ez;
        if (r2 > rHi * rHi) continue;
        fjS = lcg(fjS); double jx = x + (fjS / 4294967296.0 - 0.5) * sp * 0.3;
        fjS = lcg(fjS); double jy = y + (fjS / 4294967296.0 - 0.5) * sp * 0.3;
        fjS = lcg(fjS); double jz = z + (fjS / 4294967296.0 - 0.5) * sp * 0.3;
        if (ROCK(s, jx, jy, jz) || voxel_rock_at(s, jx, jy, jz)) continue;
        s->px[n] = (st_t)jx; s->py[n] = (st_t)jy; s->pz[n] = (st_t)jz;
        s->pvx[n] = 0; s->pvy[n] = 0; s->pvz[n] = 0; s->pflag[n] = 0; s->pcool[n] = 0;
        s->pT[n] = (st_t)s->P.Tamb;
        n++;
      }
    }
  }
  s->S.nP = n;
  memset(s->pAir, 0, sizeof(st_t) * s->S.capacity);
  memset(s->q, 0, sizeof(st_t) * s->nCells);
  s->S.heatAcc = 0;
  s->S.vaporCount = s->S.nightVaporCount = 0;
  s->gridSampleValid = 0;
  s->S.waterTopY = cy + R2;
  or_build_planet_gravity(s);
  s->S.gRamp = 0;
  or_splat_density(s);
  s->S.iso = or_autotune_iso(s);
  s->S.umax = 0;
  s->S.airborneCount = 0;
}

/* ------------------------------------------------------------ sampling
 * Face coordinates and trilinear sample, js/solver.js:737-854. */
static inline void face_coords(const or_solver* s, int comp, double x, double y, double z,
                               int* pi, int* pj, int* pk, double* ptx, double* pty, double* ptz) {
  double dx = s->dx, a, b, c;
  int nx = s->nx, ny = s->ny, nz = s->nz;
  if (comp == 0) { a = x / dx; b = y / dx - 0.5; c = z / dx - 0.5; }
  else if (comp == 1) { a = x / dx - 0.5; b = y / dx; c = z / dx - 0.5; }
  else { a = x / dx - 0.5; b = y / dx - 0.5; c = z / dx; }
  double fi = floor(a), fj = floor(b), fk = floor(c);
  if (fi < 0) { *pi = 0; *ptx = 0; } else if (fi > nx - 1) { *pi = nx - 1; *ptx = 1; } else { *pi = (int)fi; *ptx = a - fi; }
  if (fj < 0) { *pj = 0; *pty = 0; } else if (fj > ny - 2) { *pj = ny - 2; *pty = 1; } else { *pj = (int)fj; *pty = b - fj; }
  if (fk < 0) { *pk = 0; *ptz = 0; } else if (fk > nz - 2) { *pk = nz - 2; *ptz = 1; } else { *pk = (int)fk; *ptz = c - fk; }
}
static inline void face_strides(const or_solver* s, int comp, int i0, int j0, int k0,
                                long* idx, long* sj, long* sk) {
  int nx = s->nx, ny = s->ny;
  if (comp == 0) { *sj = nx + 1; *sk = (long)ny * (nx + 1); *idx = ((long)k0 * ny + j0) * (nx + 1) + i0; }
  else if (comp == 1) { *sj = nx; *sk = (long)(ny + 1) * nx; *idx = ((long)k0 * (ny + 1) + j0) * nx + i0; }
  else { *sj = nx; *sk = (long)ny * nx; *idx = ((long)k0 * ny + j0) * nx + i0; }
}
static inline double tri(const st_t* a, long idx, long sj, long sk, double tx, double ty, double tz) {
  double s0 = 1 - tx, s1 = tx, t0 = 1 - ty, t1 = ty, r0 = 1 - tz, r1 = tz;
  long o1 = idx + sj, o2 = idx + sk, o3 = o2 + sj;
  return ((a[idx] * s0 + a[idx + 1] * s1) * t0 + (a[o1] * s0 + a[o1 + 1] * s1) * t1) * r0
       + ((a[o2] * s0 + a[o2 + 1] * s1) * t0 + (a[o3] * s0 + a[o3 + 1] * s1) * t1) * r1;
}
static inline const st_t* comp_arr(const or_solver* s, int comp) {
  return comp == 0 ? s->u : (comp == 1 ? s->v : s->w);
}
static double sample_arr(const or_solver* s, const st_t* arr, int comp, double x, double y, double z) {
  int i0, j0, k0; double tx, ty, tz; long idx, sj, sk;
  face_coords(s, comp, x, y, z, &i0, &j0, &k0, &tx, &ty, &tz);
  face_strides(s, comp, i0, j0, k0, &idx, &sj, &sk);
  return tri(arr, idx, sj, sk, tx, ty, tz);
}
static void sample_vel3(const or_solver* s, double x, double y, double z, double out[3]) {
  out[0] = sample_arr(s, s->u, 0, x, y, z);
  out[1] = sample_arr(s, s->v, 1, x, y, z);
  out[2] = sample_arr(s, s->w, 2, x, y, z);
}
void or_sample_vel(or_solver* s, double x, double y, double z, double out[3]) { sample_vel3(s, x, y, z, out); }
double or_sample_face(or_solver* s, int comp, double x, double y, double z) {
  return sample_arr(s, comp_arr(s, comp), comp, x, y, z);
}

/* ------------------------------------------------------------ rasterize
 * _rasterizeStatic, js/solver.js:865-939 (no balls). */
void or_rasterize_static(or_solver* s) {
  int nx = s->nx, ny = s->ny, nz = s->nz, i, j, k;
  if (!s->staticValid) {
    double dxr = s->dx; int tvn = s->tn; double tvd = s->hasTerr ? s->tdv : 1;
    double coreR2 = s->S.coreR * s->S.coreR;
    for (k = 0; k < nz; k++) {
      double dz2 = (k + 0.5) * dxr - s->cz; dz2 *= dz2;
      for (j = 0; j < ny; j++) {
        long row = ((long)k * ny + j) * nx;
        double dy2 = (j + 0.5) * dxr - s->cy; dy2 *= dy2;
        int shell = (j == 0 || j == ny - 1 || k == 0 || k == nz - 1);
        for (i = 0; i < nx; i++) {
          int rock;
          if (s->hasTerr) {
            int vx = jtrunc((i + 0.5) * dxr / tvd), vy = jtrunc((j + 0.5) * dxr / tvd), vz = jtrunc((k + 0.5) * dxr / tvd);
            if (vx < 0) vx = 0; else if (vx >= tvn) vx = tvn - 1;
            if (vy < 0) vy = 0; else if (vy >= tvn) vy = tvn - 1;
            if (vz < 0) vz = 0; else if (vz >= tvn) vz = tvn - 1;
            rock = s->tsolid[((size_t)vz * tvn + vy) * tvn + vx] == 1;
          } else {
            double dx2 = (i + 0.5) * dxr - s->cx; dx2 *= dx2;
            rock = dx2 + dy2 + dz2 < coreR2;
          }
          s->staticTypes[row + i] = (shell || i == 0 || i == nx - 1 || rock) ? SOLID : AIR;
        }
      }
    }
    s->staticValid = 1;
  }
  memcpy(s->cellType, s->staticTypes, s->nCells);
  /* balls become moving solids, js/solver.js:918-938 */
  if (s->nBalls || s->hadSolidVelocity) {
    memset(s->svx, 0, sizeof(st_t) * s->nCells); memset(s->svy, 0, sizeof(st_t) * s->nCells);
    memset(s->svz, 0, sizeof(st_t) * s->nCells);
  }
  s->hadSolidVelocity = s->nBalls > 0;
  double dx = s->dx;
  for (int n = 0; n < s->nBalls; n++) {
    const double* b = s->balls[n];
    /* a non-finite ball covers no cell (NaN bounds, or an infinite distance) */
    if (!isfinite(b[BX]) || !isfinite(b[BY]) || !isfinite(b[BZ]) || !isfinite(b[BR])) continue;
    double r = b[BR], rr = (r + 0.4 * dx) * (r + 0.4 * dx);
    int i0 = jfloor_clamp((b[BX] - r) / dx, 1, nx - 2), i1 = jceil_clamp((b[BX] + r) / dx, 1, nx - 2);
    int j0 = jfloor_clamp((b[BY] - r) / dx, 1, ny - 2), j1 = jceil_clamp((b[BY] + r) / dx, 1, ny - 2);
    int k0 = jfloor_clamp((b[BZ] - r) / dx, 1, nz - 2), k1 = jceil_clamp((b[BZ] + r) / dx, 1, nz - 2);
    for (k = k0; k <= k1; k++) for (j = j0; j <= j1; j++) for (i = i0; i <= i1; i++) {
      double cx = (i + 0.5) * dx - b[BX], cy = (j + 0.5) * dx - b[BY], cz = (k + 0.5) * dx - b[BZ];
      if (cx * cx + cy * cy + cz * cz <= rr) {
        long ci = ((long)k * ny + j) * nx + i;
        s->cellType[ci] = SOLID;
        s->svx[ci] = (st_t)b[BVX]; s->svy[ci] = (st_t)b[BVY]; s->svz[ci] = (st_t)b[BVZ];
      }
    }
  }
}

/* _markFluidCells, js/solver.js:945-1000 */
void or_mark_fluid(or_solver* s) {
  int nx = s->nx, ny = s->ny, nz = s->nz, nP = s->S.nP, p, i, j, k;
  double dx = s->dx, oceanR = s->S.oceanR;
  int jTop = ny - 2;
  double skyAlt = 2 * dx > 0.3 ? 2 * dx : 0.3;
  for (p = 0; p < nP; p++) {
    if (s->pflag[p] != 0) continue;
    double X = s->px[p], Y = s->py[p], Z = s->pz[p];
    double rx = X - s->cx, ry = Y - s->cy, rz = Z - s->cz;
    double radius2 = rx * rx + ry * ry + rz * rz;
    if (radius2 > (oceanR + 0.3) * (oceanR + 0.3) &&
        sqrt(radius2) - TRAD(s, X, Y, Z) > skyAlt &&
        !ROCK(s, X, Y, Z)) {
      s->pflag[p] = 1; continue;
    }
    i = jfloor_clamp(X / dx, 0, nx - 1);
    j = jfloor_clamp(Y / dx, 0, ny - 1);
    k = jfloor_clamp(Z / dx, 0, nz - 1);
    if (j >= jTop) {
      double jx = X - s->cx, jy = Y - s->cy, jz = Z - s->cz;
      if (sqrt(jx * jx + jy * jy + jz * jz) - TRAD(s, X, Y, Z) > 0.3) { s->pflag[p] = 1; continue; }
    }
    long idx = ((long)k * ny + j) * nx + i;
    if (s->cellType[idx] == AIR) s->cellType[idx] = FLUID;
  }
}

/* ------------------------------------------------------------ P2G
 * _p2gInto + _p2gNormalizeFace, js/solver.js:1035-1120 */
void or_clear_faces(or_solver* s) {
  memset(s->u, 0, sizeof(st_t) * s->uN); memset(s->v, 0, sizeof(st_t) * s->vN); memset(s->w, 0, sizeof(st_t) * s->wN);
  memset(s->uW, 0, sizeof(st_t) * s->uN); memset(s->vW, 0, sizeof(st_t) * s->vN); memset(s->wW, 0, sizeof(st_t) * s->wN);
}
static inline void p2g_comp(or_solver* s, int comp, st_t* A, st_t* Wt, double x, double y, double z, double vel) {
  int i0, j0, k0; double tx, ty, tz; long idx, sj, sk;
  face_coords(s, comp, x, y, z, &i0, &j0, &k0, &tx, &ty, &tz);
  face_strides(s, comp, i0, j0, k0, &idx, &sj, &sk);
  double s0 = 1 - tx, s1 = tx, t0 = 1 - ty, t1 = ty, r0 = 1 - tz, r1 = tz;
  double wA = s0 * t0, wB = s1 * t0, wC = s0 * t1, wD = s1 * t1;
  A[idx] += wA * r0 * vel; Wt[idx] += wA * r0;
  A[idx + 1] += wB * r0 * vel; Wt[idx + 1] += wB * r0;
  A[idx + sj] += wC * r0 * vel; Wt[idx + sj] += wC * r0;
  A[idx + sj + 1] += wD * r0 * vel; Wt[idx + sj + 1] += wD * r0;
  A[idx + sk] += wA * r1 * vel; Wt[idx + sk] += wA * r1;
  A[idx + sk + 1] += wB * r1 * vel; Wt[idx + sk + 1] += wB * r1;
  A[idx + sk + sj] += wC * r1 * vel; Wt[idx + sk + sj] += wC * r1;
  A[idx + sk + sj + 1] += wD * r1 * vel; Wt[idx + sk + sj + 1] += wD * r1;
}
void or_p2g(or_solver* s) {
  int p, nP = s->S.nP;
  for (p = 0; p < nP; p++) {
    if (s->pflag[p] != 0) continue;
    double x = s->px[p], y = s->py[p], z = s->pz[p];
    p2g_comp(s, 0, s->u, s->uW, x, y, z, s->pvx[p]);
    p2g_comp(s, 1, s->v, s->vW, x, y, z, s->pvy[p]);
    p2g_comp(s, 2, s->w, s->wW, x, y, z, s->pvz[p]);
  }
  long i;
  for (i = 0; i < s->uN; i++) if (s->uW[i] > 1e-8) s->u[i] /= s->uW[i];
  for (i = 0; i < s->vN; i++) if (s->vW[i] > 1e-8) s->v[i] /= s->vW[i];
  for (i = 0; i < s->wN; i++) if (s->wW[i] > 1e-8) s->w[i] /= s->wW[i];
}

/* ------------------------------------------------------------ BC
 * _applyBCSlice, js/solver.js:1130-1171 (no moving solids: sv = 0) */
void or_apply_bc(or_solver* s) {
  int nx = s->nx, ny = s->ny, nz = s->nz, i, j, k;
  st_t *u = s->u, *v = s->v, *w = s->w; const uint8_t* type = s->cellType;
  for (k = 0; k < nz; k++) for (j = 0; j < ny; j++) {
    u[((long)k * ny + j) * (nx + 1)] = 0;
    u[((long)k * ny + j) * (nx + 1) + nx] = 0;
  }
  for (k = 0; k < nz; k++) for (i = 0; i < nx; i++) {
    v[((long)k * (ny + 1)) * nx + i] = 0;
    v[((long)k * (ny + 1) + ny) * nx + i] = 0;
  }
  for (j = 0; j < ny; j++) for (i = 0; i < nx; i++) w[(long)j * nx + i] = 0;
  for (j = 0; j < ny; j++) for (i = 0; i < nx; i++) w[((long)nz * ny + j) * nx + i] = 0;
  for (k = 0; k < nz; k++) for (j = 0; j < ny; j++) for (i = 1; i < nx; i++) {
    long c = ((long)k * ny + j) * nx + i;
    int cL = type[c - 1], cR = type[c];
    long idx = ((long)k * ny + j) * (nx + 1) + i;
    if (cL == SOLID) u[idx] = s->svx[c - 1]; else if (cR == SOLID) u[idx] = s->svx[c];
  }
  for (k = 0; k < nz; k++) for (j = 1; j < ny; j++) for (i = 0; i < nx; i++) {
    long c = ((long)k * ny + j) * nx + i;
    int cL = type[c - nx], cR = type[c];
    long idx = ((long)k * (ny + 1) + j) * nx + i;
    if (cL == SOLID) v[idx] = s->svy[c - nx]; else if (cR == SOLID) v[idx] = s->svy[c];
  }
  for (k = 1; k < nz; k++) for (j = 0; j < ny; j++) for (i = 0; i < nx; i++) {
    long c = ((long)k * ny + j) * nx + i;
    int cL = type[c - (long)nx * ny], cR = type[c];
    if (cL == SOLID) w[c] = s->svz[c - (long)nx * ny]; else if (cR == SOLID) w[c] = s->svz[c];
  }
}

void or_snapshot_old(or_solver* s) {                         /* js/solver.js:2579 */
  memcpy(s->uO, s->u, sizeof(st_t) * s->uN);
  memcpy(s->vO, s->v, sizeof(st_t) * s->vN);
  memcpy(s->wO, s->w, sizeof(st_t) * s->wN);
}

/* ------------------------------------------------------------ gravity
 * _buildPlanetGravity, js/solver.js:1177-1210 */
void or_build_planet_gravity(or_solver* s) {
  int nx = s->nx, ny = s->ny, nz = s->nz, i, j, k; double dx = s->dx;
  double cx = s->cx, cy = s->cy, cz = s->cz, g0 = s->S.oceanR * s->S.oceanR;
  if (!s->hasGravity) {
    s->gu = xcalloc(s->uN, sizeof(st_t)); s->gv = xcalloc(s->vN, sizeof(st_t)); s->gw = xcalloc(s->wN, sizeof(st_t));
    s->hasGravity = 1;
  }
  for (k = 0; k < nz; k++) for (j = 0; j < ny; j++) {
    double ey = (j + 0.5) * dx - cy, ez = (k + 0.5) * dx - cz;
    for (i = 0; i <= nx; i++) {
      double ex = i * dx - cx;
      double r3 = pow(ex * ex + ey * ey + ez * ez, 1.5); if (r3 == 0) r3 = 1e-9;
      s->gu[((long)k * ny + j) * (nx + 1) + i] = (st_t)(-g0 * ex / r3);
    }
  }
  for (k = 0; k < nz; k++) for (j = 0; j <= ny; j++) {
    double ey2 = j * dx - cy, ez2 = (k + 0.5) * dx - cz;
    for (i = 0; i < nx; i++) {
      double exx = (i + 0.5) * dx - cx;
      double r32 = pow(exx * exx + ey2 * ey2 + ez2 * ez2, 1.5); if (r32 == 0) r32 = 1e-9;
      s->gv[((long)k * (ny + 1) + j) * nx + i] = (st_t)(-g0 * ey2 / r32);
    }
  }
  for (k = 0; k <= nz; k++) for (j = 0; j < ny; j++) {
    double ey3 = (j + 0.5) * dx - cy, ez3 = k * dx - cz;
    for (i = 0; i < nx; i++) {
      double ex3 = (i + 0.5) * dx - cx;
      double r33 = pow(ex3 * ex3 + ey3 * ey3 + ez3 * ez3, 1.5); if (r33 == 0) r33 = 1e-9;
      s->gw[((long)k * ny + j) * nx + i] = (st_t)(-g0 * ez3 / r33);
    }
  }
}

/* _applyPlanetGravity (serial wrapper js/solver.js:2656-2662, which
 * overrides :1217-1225) + _applyPlanetGravitySlice :1229-1256 */
void or_planet_gravity(or_solver* s, double dt) {
  if (!s->hasGravity) return;
  double gs = s->S.gRamp / 1.5; if (gs > 1) gs = 1;
  s->S.gRamp += dt;
  if (gs <= 0) return;
  gs *= s->P.gravity;
  if (gs <= 0) return;
  int nx = s->nx, ny = s->ny, nz = s->nz, i, j, k; const uint8_t* type = s->cellType;
  for (k = 0; k < nz; k++) for (j = 0; j < ny; j++) {
    long base = (long)k * ny + j, row = base * nx;
    for (i = 1; i < nx; i++) {
      int cL = type[row + i - 1], cR = type[row + i];
      if (cL == FLUID || cR == FLUID) { long idx = base * (nx + 1) + i; s->u[idx] += s->gu[idx] * dt * gs; }
    }
  }
  for (k = 0; k < nz; k++) for (j = 1; j < ny; j++) {
    long row2 = ((long)k * (ny + 1) + j) * nx;
    for (i = 0; i < nx; i++) {
      int cL = type[((long)k * ny + j - 1) * nx + i], cR = type[((long)k * ny + j) * nx + i];
      if (cL == FLUID || cR == FLUID) { long idx = row2 + i; s->v[idx] += s->gv[idx] * dt * gs; }
    }
  }
  for (k = 1; k < nz; k++) for (j = 0; j < ny; j++) {
    long row3 = ((long)k * ny + j) * nx;
    for (i = 0; i < nx; i++) {
      int cL = type[((long)(k - 1) * ny + j) * nx + i], cR = type[row3 + i];
      if (cL == FLUID || cR == FLUID) { long idx = row3 + i; s->w[idx] += s->gw[idx] * dt * gs; }
    }
  }
}

/* ------------------------------------------------------------ viscosity
 * _viscosity, js/solver.js:1259-1304. viscJacobi=1 reads neighbours from the
 * uO/vO/wO snapshot (equal to u/v/w on entry) instead of the partially
 * updated arrays; the two orders differ by O(coef^2). */
void or_viscosity(or_solver* s, double dt) {
  double nu = s->P.viscosity;
  if (nu <= 1e-6) return;
  int nx = s->nx, ny = s->ny, nz = s->nz, i, j, k; double dx = s->dx; const uint8_t* type = s->cellType;
  double coef = jmin(nu * dt / (dx * dx), 0.24);
  int jac = s->P.viscJacobi;
  const st_t *ru = jac ? s->uO : s->u, *rv = jac ? s->vO : s->v, *rw = jac ? s->wO : s->w;
  for (k = 0; k < nz; k++) for (j = 0; j < ny; j++) for (i = 1; i < nx; i++) {
    if (type[((long)k * ny + j) * nx + i - 1] != FLUID || type[((long)k * ny + j) * nx + i] != FLUID) continue;
    long idx = ((long)k * ny + j) * (nx + 1) + i;
    double val = (double)ru[idx] * 6;
    val -= (i - 1 >= 0) ? ru[idx - 1] : ru[idx];
    val -= (i + 1 <= nx) ? ru[idx + 1] : ru[idx];
    val -= (j - 1 >= 0) ? ru[idx - (nx + 1)] : ru[idx];
    val -= (j + 1 < ny) ? ru[idx + (nx + 1)] : ru[idx];
    val -= (k - 1 >= 0) ? ru[idx - (long)ny * (nx + 1)] : ru[idx];
    val -= (k + 1 < nz) ? ru[idx + (long)ny * (nx + 1)] : ru[idx];
    s->u[idx] = (st_t)(ru[idx] + coef * val);
  }
  for (k = 0; k < nz; k++) for (j = 1; j < ny; j++) for (i = 0; i < nx; i++) {
    if (type[((long)k * ny + j - 1) * nx + i] != FLUID || type[((long)k * ny + j) * nx + i] != FLUID) continue;
    long idx = ((long)k * (ny + 1) + j) * nx + i;
    double val = (double)rv[idx] * 6;
    val -= (i - 1 >= 0) ? rv[idx - 1] : rv[idx];
    val -= (i + 1 < nx) ? rv[idx + 1] : rv[idx];
    val -= (j - 1 >= 0) ? rv[idx - nx] : rv[idx];
    val -= (j + 1 <= ny) ? rv[idx + nx] : rv[idx];
    val -= (k - 1 >= 0) ? rv[idx - (long)(ny + 1) * nx] : rv[idx];
    val -= (k + 1 < nz) ? rv[idx + (long)(ny + 1) * nx] : rv[idx];
    s->v[idx] = (st_t)(rv[idx] + coef * val);
  }
  for (k = 1; k < nz; k++) for (j = 0; j < ny; j++) for (i = 0; i < nx; i++) {
    if (type[((long)(k - 1) * ny + j) * nx + i] != FLUID || type[((long)k * ny + j) * nx + i] != FLUID) continue;
    long idx = ((long)k * ny + j) * nx + i;
    double val = (double)rw[idx] * 6;
    val -= (i - 1 >= 0) ? rw[idx - 1] : rw[idx];
    val -= (i + 1 < nx) ? rw[idx + 1] : rw[idx];
    val -= (j - 1 >= 0) ? rw[idx - nx] : rw[idx];
    val -= (j + 1 < ny) ? rw[idx + nx] : rw[idx];
    val -= (k - 1 >= 0) ? rw[idx - (long)ny * nx] : rw[idx];
    val -= (k + 1 <= nz) ? rw[idx + (long)ny * nx] : rw[idx];
    s->w[idx] = (st_t)(rw[idx] + coef * val);
  }
}

/* ------------------------------------------------------------ pressure
 * _pressureSolve, js/solver.js:1312-1410. sorRedBlack=1 sweeps the cells of
 * colour (i+j+k)&1 == 0 first, then colour 1 — one iteration is both
 * colours. sorTol>0 iterates to ||b-Aq||/||b|| <= sorTol (checked every
 * sorCheckEvery iterations, capped at sorMaxIters); otherwise pressureIters. */
static double residual_impl(or_solver* s) {
  int nF = s->nFluid, fi; double rr = 0, bb = 0;
  for (fi = 0; fi < nF; fi++) {
    int c = s->fluidList[fi];
    double sum = 0;
    for (int a = s->pStart[fi]; a < s->pStart[fi + 1]; a++) sum += s->q[s->pAdj[a]];
    double r = (double)s->rhs[c] + sum - (double)s->diag[c] * s->q[c];
    rr += r * r; bb += (double)s->rhs[c] * s->rhs[c];
  }
  return bb > 0 ? sqrt(rr) / sqrt(bb) : sqrt(rr);
}
double or_residual(or_solver* s) { return s->nFluid > 0 && s->pStart ? residual_impl(s) : 0; }

void or_pressure_solve(or_solver* s) {
  int nx = s->nx, ny = s->ny, nz = s->nz, i, j, k, c, fi, nF = 0; double dx = s->dx;
  const uint8_t* type = s->cellType;
  for (k = 0; k < nz; k++) for (j = 0; j < ny; j++) {
    long row = (long)k * ny + j;
    for (i = 0; i < nx; i++) {
      c = (int)(row * nx + i);
      if (type[c] != FLUID) { s->q[c] = 0; continue; }
      s->fluidList[nF++] = c;
    }
  }
  s->S.sorIters = 0; s->S.sorRelRes = 0;
  if (nF == 0) { memcpy(s->cellPhi, s->q, sizeof(st_t) * s->nCells); s->nFluid = 0; return; }
  s->nFluid = nF;
  int nxy = nx * ny;
  for (fi = 0; fi < nF; fi++) {
    c = s->fluidList[fi];
    i = c % nx; j = (c / nx) % ny; k = c / nxy;
    long r6 = (long)c * 6; int Nf = 0, Na = 0, d;
    int cm = i > 0 ? c - 1 : -1, cp = i < nx - 1 ? c + 1 : -1;
    int cd = j > 0 ? c - nx : -1, cu = j < ny - 1 ? c + nx : -1;
    int cb = k > 0 ? c - nxy : -1, cf = k < nz - 1 ? c + nxy : -1;
    for (d = 0; d < 6; d++) {
      int n = d == 0 ? cm : d == 1 ? cp : d == 2 ? cd : d == 3 ? cu : d == 4 ? cb : cf;
      if (n < 0) { s->nb[r6 + d] = -1; continue; }
      int t = type[n];
      if (t == FLUID) { s->nb[r6 + d] = n; Nf++; }
      else if (t == AIR) { s->nb[r6 + d] = -1; Na++; }
      else s->nb[r6 + d] = -1;
    }
    s->diag[c] = (st_t)(Nf + Na);
    double div = ((double)s->u[((long)k * ny + j) * (nx + 1) + i + 1] - s->u[((long)k * ny + j) * (nx + 1) + i] +
                  s->v[((long)k * (ny + 1) + j + 1) * nx + i] - s->v[((long)k * (ny + 1) + j) * nx + i] +
                  s->w[((long)(k + 1) * ny + j) * nx + i] - s->w[((long)k * ny + j) * nx + i]) / dx;
    s->rhs[c] = (st_t)(-dx * dx * div);
  }
  double omega = s->P.omega, om1 = 1 - omega;
  if (s->pCap < nF + 1) {
    free(s->pStart); free(s->pAdj); free(s->pW);
    s->pStart = xcalloc(nF + 1, sizeof(int32_t)); s->pAdj = xcalloc((size_t)6 * nF, sizeof(int32_t));
    s->pW = xcalloc(nF, sizeof(st_t)); s->pCap = nF + 1;
  }
  int na = 0;
  for (fi = 0; fi < nF; fi++) {
    s->pStart[fi] = na;
    c = s->fluidList[fi];
    long r6 = (long)c * 6;
    for (int d2 = 0; d2 < 6; d2++) { int nn = s->nb[r6 + d2]; if (nn >= 0) s->pAdj[na++] = nn; }
    double dgW = s->diag[c];
    s->pW[fi] = (st_t)(dgW > 0 ? omega / dgW : 0);
  }
  s->pStart[nF] = na;
  st_t* q = s->q;
  int rb = s->P.sorRedBlack;
  int tolMode = s->P.sorTol > 0;
  int iters = tolMode ? s->P.sorMaxIters : s->P.pressureIters;
  int check = s->P.sorCheckEvery > 0 ? s->P.sorCheckEvery : 1;
  int it; double rel = -1;
  for (it = 0; it < iters; it++) {
    if (!rb) {
      for (fi = 0; fi < nF; fi++) {
        double sum = 0;
        for (int ai = s->pStart[fi], ae = s->pStart[fi + 1]; ai < ae; ai++) sum += q[s->pAdj[ai]];
        c = s->fluidList[fi];
        q[c] = (st_t)(q[c] * om1 + s->pW[fi] * (s->rhs[c] + sum));
      }
    } else {
      for (int color = 0; color < 2; color++) {
        for (fi = 0; fi < nF; fi++) {
          c = s->fluidList[fi];
          i = c % nx; j = (c / nx) % ny; k = c / nxy;
          if (((i + j + k) & 1) != color) continue;
          double sum = 0;
          for (int ai = s->pStart[fi], ae = s->pStart[fi + 1]; ai < ae; ai++) sum += q[s->pAdj[ai]];
          q[c] = (st_t)(q[c] * om1 + s->pW[fi] * (s->rhs[c] + sum));
        }
      }
    }
    if (tolMode && ((it + 1) % check == 0)) {
      rel = residual_impl(s);
      if (rel <= s->P.sorTol) { it++; break; }
    }
  }
  (void)rel;
  s->S.sorIters = it;
  s->S.sorRelRes = residual_impl(s);
  memcpy(s->cellPhi, q, sizeof(st_t) * s->nCells);
}

/* _projectSlice, js/solver.js:1417-1443 */
void or_project(or_solver* s) {
  int nx = s->nx, ny = s->ny, nz = s->nz, i, j, k; double inv = 1 / s->dx;
  const uint8_t* type = s->cellType; const st_t* phi = s->cellPhi;
  for (k = 0; k < nz; k++) for (j = 0; j < ny; j++) for (i = 1; i < nx; i++) {
    long c = ((long)k * ny + j) * nx + i;
    int cL = type[c - 1], cR = type[c];
    if (cL == SOLID || cR == SOLID) continue;
    double pL = cL == FLUID ? phi[c - 1] : 0, pR = cR == FLUID ? phi[c] : 0;
    s->u[((long)k * ny + j) * (nx + 1) + i] -= (pR - pL) * inv;
  }
  for (k = 0; k < nz; k++) for (j = 1; j < ny; j++) for (i = 0; i < nx; i++) {
    long c = ((long)k * ny + j) * nx + i;
    int cL = type[c - nx], cR = type[c];
    if (cL == SOLID || cR == SOLID) continue;
    double pL = cL == FLUID ? phi[c - nx] : 0, pR = cR == FLUID ? phi[c] : 0;
    s->v[((long)k * (ny + 1) + j) * nx + i] -= (pR - pL) * inv;
  }
  for (k = 1; k < nz; k++) for (j = 0; j < ny; j++) for (i = 0; i < nx; i++) {
    long c = ((long)k * ny + j) * nx + i;
    int cL = type[c - (long)nx * ny], cR = type[c];
    if (cL == SOLID || cR == SOLID) continue;
    double pL = cL == FLUID ? phi[c - (long)nx * ny] : 0, pR = cR == FLUID ? phi[c] : 0;
    s->w[c] -= (pR - pL) * inv;
  }
}

/* _vorticityConfinement, js/solver.js:1454-1559 */
void or_vorticity(or_solver* s, double dt) {
  double eps = s->P.vorticity;
  if (!(eps > 0)) return;
  int nx = s->nx, ny = s->ny, nz = s->nz, i, j, k; long c; long nxy = (long)nx * ny;
  const uint8_t* type = s->cellType; st_t *u = s->u, *v = s->v, *w = s->w;
  st_t *cx = s->vcx, *cy = s->vcy, *cz = s->vcz, *omg = s->omg, *ox = s->omx, *oy = s->omy, *oz = s->omz;
  for (k = 0; k < nz; k++) for (j = 0; j < ny; j++) {
    long rowC = ((long)k * ny + j) * nx, rowU = ((long)k * ny + j) * (nx + 1), rowV = ((long)k * (ny + 1) + j) * nx;
    for (i = 0; i < nx; i++) {
      c = rowC + i;
      cx[c] = (st_t)(0.5 * ((double)u[rowU + i] + u[rowU + i + 1]));
      cy[c] = (st_t)(0.5 * ((double)v[rowV + i] + v[rowV + nx + i]));
      cz[c] = (st_t)(0.5 * ((double)w[rowC + i] + w[rowC + nxy + i]));
    }
  }
  double inv2 = 0.5 / s->dx;
  for (k = 0; k < nz; k++) for (j = 0; j < ny; j++) {
    long row = ((long)k * ny + j) * nx;
    for (i = 0; i < nx; i++) {
      c = row + i;
      long im = i > 0 ? c - 1 : c, ip = i < nx - 1 ? c + 1 : c;
      long jm = j > 0 ? c - nx : c, jp = j < ny - 1 ? c + nx : c;
      long km = k > 0 ? c - nxy : c, kp = k < nz - 1 ? c + nxy : c;
      double wx = ((double)cz[jp] - cz[jm] - ((double)cy[kp] - cy[km])) * inv2;
      double wy = ((double)cx[kp] - cx[km] - ((double)cz[ip] - cz[im])) * inv2;
      double wz = ((double)cy[ip] - cy[im] - ((double)cx[jp] - cx[jm])) * inv2;
      ox[c] = (st_t)wx; oy[c] = (st_t)wy; oz[c] = (st_t)wz;
      omg[c] = (st_t)sqrt(wx * wx + wy * wy + wz * wz);
    }
  }
  double fCap = 6.0, omFloor = 0.35; int nF = s->nFluid, fi;
  for (fi = 0; fi < nF; fi++) {
    c = s->fluidList[fi];
    i = (int)(c % nx); j = (int)((c / nx) % ny); k = (int)(c / nxy);
    if (omg[c] < omFloor ||
        (i > 0 && type[c - 1] != FLUID) || (i < nx - 1 && type[c + 1] != FLUID) ||
        (j > 0 && type[c - nx] != FLUID) || (j < ny - 1 && type[c + nx] != FLUID) ||
        (k > 0 && type[c - nxy] != FLUID) || (k < nz - 1 && type[c + nxy] != FLUID)) {
      cx[c] = 0; cy[c] = 0; cz[c] = 0; continue;
    }
    double gx = (double)omg[i < nx - 1 ? c + 1 : c] - omg[i > 0 ? c - 1 : c];
    double gy = (double)omg[j < ny - 1 ? c + nx : c] - omg[j > 0 ? c - nx : c];
    double gz = (double)omg[k < nz - 1 ? c + nxy : c] - omg[k > 0 ? c - nxy : c];
    double g2 = gx * gx + gy * gy + gz * gz;
    if (g2 < 1e-12) { cx[c] = 0; cy[c] = 0; cz[c] = 0; continue; }
    double inv = 1 / sqrt(g2);
    double Nx = gx * inv, Ny = gy * inv, Nz = gz * inv;
    double fx = eps * (Ny * oz[c] - Nz * oy[c]);
    double fy = eps * (Nz * ox[c] - Nx * oz[c]);
    double fz = eps * (Nx * oy[c] - Ny * ox[c]);
    double f2 = fx * fx + fy * fy + fz * fz;
    if (f2 > fCap * fCap) { double fs = fCap / sqrt(f2); fx *= fs; fy *= fs; fz *= fs; }
    cx[c] = (st_t)(fx * dt); cy[c] = (st_t)(fy * dt); cz[c] = (st_t)(fz * dt);
  }
  for (fi = 0; fi < nF; fi++) {
    c = s->fluidList[fi];
    i = (int)(c % nx); j = (int)((c / nx) % ny); k = (int)(c / nxy);
    if (i < nx - 1 && type[c + 1] == FLUID)
      u[((long)k * ny + j) * (nx + 1) + i + 1] += 0.5 * ((double)cx[c] + cx[c + 1]);
    if (j < ny - 1 && type[c + nx] == FLUID)
      v[((long)k * (ny + 1) + j + 1) * nx + i] += 0.5 * ((double)cy[c] + cy[c + nx]);
    if (k < nz - 1 && type[c + nxy] == FLUID)
      w[((long)(k + 1) * ny + j) * nx + i] += 0.5 * ((double)cz[c] + cz[c + nxy]);
  }
}

/* _clampUmSlice, js/solver.js:2629-2653 */
double or_clamp_um(or_solver* s) {
  double vcap = s->P.maxSpeed * 1.1, um = 0, av; long i;
  st_t* arrs[3] = { s->u, s->v, s->w }; long ns[3] = { s->uN, s->vN, s->wN };
  for (int cmp = 0; cmp < 3; cmp++) {
    st_t* a = arrs[cmp];
    for (i = 0; i < ns[cmp]; i++) {
      if (a[i] > vcap) a[i] = (st_t)vcap; else if (a[i] < -vcap) a[i] = (st_t)(-vcap);
      av = a[i]; if (av > um) um = av; else if (-av > um) um = -av;
    }
  }
  return um;
}

/* _extrapolate, js/solver.js:1562-1636. extrapJacobi=1 counts only faces
 * valid before the pass (the reference's in-place pass also counts faces
 * filled earlier in the same pass, in lexicographic order). */
void or_extrapolate(or_solver* s) {
  int nx = s->nx, ny = s->ny, nz = s->nz; long nxy = (long)nx * ny;
  const uint8_t* type = s->cellType;
  int jac = s->P.extrapJacobi;
  for (int ci = 0; ci < 3; ci++) {
    st_t* arr = ci == 0 ? s->u : ci == 1 ? s->v : s->w;
    const st_t* wgt = ci == 0 ? s->uW : ci == 1 ? s->vW : s->wW;
    uint8_t* valid = ci == 0 ? s->validU : ci == 1 ? s->validV : s->validW;
    int d0 = ci == 0 ? nx + 1 : nx, d1 = ci == 1 ? ny + 1 : ny, d2 = ci == 2 ? nz + 1 : nz;
    long N = (long)d0 * d1 * d2, idx; int i, j, k;
    for (k = 0; k < d2; k++) {
      long kc = (long)k * ny;
      for (j = 0; j < d1; j++) {
        long base = ((long)k * d1 + j) * d0, rowC = (kc + j) * nx;
        for (i = 0; i < d0; i++) {
          idx = base + i; int solidAdj;
          if (ci == 0) {
            solidAdj = i == 0 || i == nx;
            if (!solidAdj) { long cl = rowC + i - 1; solidAdj = type[cl] == SOLID || type[cl + 1] == SOLID; }
          } else if (ci == 1) {
            solidAdj = j == 0 || j == ny;
            if (!solidAdj) solidAdj = type[rowC - nx + i] == SOLID || type[rowC + i] == SOLID;
          } else {
            solidAdj = k == 0 || k == nz;
            if (!solidAdj) solidAdj = type[rowC - nxy + i] == SOLID || type[rowC + i] == SOLID;
          }
          valid[idx] = (wgt[idx] > 1e-8 || solidAdj) ? 1 : 0;
        }
      }
    }
    long sK = (long)d0 * d1;
    for (k = 0; k < d2; k++) {
      int kLo = k > 0, kHi = k < d2 - 1;
      for (j = 0; j < d1; j++) {
        long base2 = ((long)k * d1 + j) * d0; int jLo = j > 0, jHi = j < d1 - 1;
        for (i = 0; i < d0; i++) {
          idx = base2 + i;
          if (valid[idx]) continue;
          double sum = 0; int cnt = 0;
#define OK_(n_) (jac ? valid[n_] == 1 : valid[n_] != 0)
          if (i > 0 && OK_(idx - 1)) { sum += arr[idx - 1]; cnt++; }
          if (i < d0 - 1 && OK_(idx + 1)) { sum += arr[idx + 1]; cnt++; }
          if (jLo && OK_(idx - d0)) { sum += arr[idx - d0]; cnt++; }
          if (jHi && OK_(idx + d0)) { sum += arr[idx + d0]; cnt++; }
          if (kLo && OK_(idx - sK)) { sum += arr[idx - sK]; cnt++; }
          if (kHi && OK_(idx + sK)) { sum += arr[idx + sK]; cnt++; }
#undef OK_
          if (cnt > 0) { arr[idx] = (st_t)(sum / cnt); valid[idx] = 2; }
        }
      }
    }
    for (idx = 0; idx < N; idx++) if (valid[idx] == 2) valid[idx] = 1;
  }
}

/* ------------------------------------------------------------ G2P
 * _g2pChunk, js/solver.js:1646-1756 */
void or_g2p(or_solver* s, double dt) {
  int nx = s->nx, ny = s->ny, nz = s->nz, nP = s->S.nP, p, airCount = 0;
  double dx = s->dx, pic = s->P.pic, maxSpeed = s->P.maxSpeed;
  const uint8_t* type = s->cellType;
  for (p = 0; p < nP; p++) {
    if (s->pflag[p] != 0) { airCount++; continue; }
    if (s->pcool[p] > 0) {
      s->pcool[p]--;
      double gdt = dt; if (gdt == 0) gdt = s->S.dtLast; if (gdt == 0) gdt = 0.01;
      s->pvy[p] = (st_t)(s->pvy[p] - s->P.gravity * gdt);
      double t3[3]; sample_vel3(s, s->px[p], s->py[p], s->pz[p], t3);
      s->advU[p] = t3[0]; s->advV[p] = t3[1]; s->advW[p] = t3[2];
      continue;
    }
    double x = s->px[p], y = s->py[p], z = s->pz[p];
    double ou = sample_arr(s, s->uO, 0, x, y, z), nu = sample_arr(s, s->u, 0, x, y, z);
    double ov = sample_arr(s, s->vO, 1, x, y, z), nv = sample_arr(s, s->v, 1, x, y, z);
    double ow = sample_arr(s, s->wO, 2, x, y, z), nw = sample_arr(s, s->w, 2, x, y, z);
    s->advU[p] = nu; s->advV[p] = nv; s->advW[p] = nw;
    s->pvx[p] = (st_t)((s->pvx[p] + nu - ou) * (1 - pic) + nu * pic);
    s->pvy[p] = (st_t)((s->pvy[p] + nv - ov) * (1 - pic) + nv * pic);
    s->pvz[p] = (st_t)((s->pvz[p] + nw - ow) * (1 - pic) + nw * pic);
    double pv2 = (double)s->pvx[p] * s->pvx[p] + (double)s->pvy[p] * s->pvy[p] + (double)s->pvz[p] * s->pvz[p];
    if (pv2 > maxSpeed * maxSpeed) {
      double psc = maxSpeed / sqrt(pv2);
      s->pvx[p] *= psc; s->pvy[p] *= psc; s->pvz[p] *= psc;
    }
    int ci = jfloor_clamp(x / dx, 0, nx - 1), cj = jfloor_clamp(y / dx, 0, ny - 1), ck = jfloor_clamp(z / dx, 0, nz - 1);
    long c = ((long)ck * ny + cj) * nx + ci;
    if (type[c] == AIR) {
      int fluidNbr =
        (ci > 0 && type[c - 1] == FLUID) || (ci < nx - 1 && type[c + 1] == FLUID) ||
        (cj > 0 && type[c - nx] == FLUID) || (cj < ny - 1 && type[c + nx] == FLUID) ||
        (ck > 0 && type[c - (long)nx * ny] == FLUID) || (ck < nz - 1 && type[c + (long)nx * ny] == FLUID);
      if (!fluidNbr && !on_rock_below(s, x, y, z)) { s->pflag[p] = 1; airCount++; }
    }
  }
  s->S.airborneCount = airCount;
  s->gridSampleValid = 1;
}

/* ------------------------------------------------------------ advection
 * _advectChunk, js/solver.js:1769-2292 (sphere mode) */
void or_advect(or_solver* s, double dt) {
  int nx = s->nx, ny = s->ny, nz = s->nz, nP = s->S.nP, p;
  double dx = s->dx, g = s->P.gravity, maxSpeed = s->P.maxSpeed, oceanR = s->S.oceanR;
  const uint8_t* type = s->cellType;
  double xLo = dx * 1.02, xHi = s->W - dx * 1.02, yLo = dx * 1.02, yHi = s->H - dx * 1.02;
  double zLo = dx * 1.02, zHi = s->D - dx * 1.02;
  double cx = s->cx, cy = s->cy, cz = s->cz;
  double domHi = s->domainR - dx * 0.02;
  double coreLo = s->S.coreR + dx * 1.02;
  int hasTerr = s->hasTerr;
  double windSX = 1, windSY = 0, windSZ = 0;
  if (s->P.hasSun) {
    windSX = s->P.sunPos[0] - cx; windSY = s->P.sunPos[1] - cy; windSZ = s->P.sunPos[2] - cz;
    double windLen = sqrt(windSX * windSX + windSY * windSY + windSZ * windSZ); if (windLen == 0) windLen = 1;
    windSX /= windLen; windSY /= windLen; windSZ /= windLen;
  }
  double rainTe = jmin(s->P.rainT, s->P.cloudT - 0.02); if (rainTe < 0) rainTe = 0;
  st_t *px = s->px, *py = s->py, *pz = s->pz, *pvx = s->pvx, *pvy = s->pvy, *pvz = s->pvz, *pAir = s->pAir;
  uint8_t *fl = s->pflag, *pcool = s->pcool;
  for (p = 0; p < nP; p++) {
    double x = px[p], y = py[p], z = pz[p];
    double vx = pvx[p], vy = pvy[p], vz = pvz[p];
    if (fl[p] == 5) {                                              /* ice, :1797-1864 */
      if (pAir[p] == 1 || !hasTerr) { pvx[p] = 0; pvy[p] = 0; pvz[p] = 0; continue; }
      double dragK = 12, gI = s->P.gravity; if (gI == 0) gI = 9.81;
      double exI = x - cx, eyI = y - cy, ezI = z - cz;
      double elI = sqrt(exI * exI + eyI * eyI + ezI * ezI); if (elI == 0) elI = 1e-9;
      double axI = -gI * 0.6 * exI / elI, ayI = -gI * 0.6 * eyI / elI, azI = -gI * 0.6 * ezI / elI;
      pvx[p] += (axI - dragK * pvx[p]) * dt;
      pvy[p] += (ayI - dragK * pvy[p]) * dt;
      pvz[p] += (azI - dragK * pvz[p]) * dt;
      x += pvx[p] * dt; y += pvy[p] * dt; z += pvz[p] * dt;
      double rrI = sqrt((x - cx) * (x - cx) + (y - cy) * (y - cy) + (z - cz) * (z - cz));
      if (rrI > oceanR + s->P.atmosphereH) {
        double scI = (oceanR + s->P.atmosphereH) / rrI;
        x = cx + (x - cx) * scI; y = cy + (y - cy) * scI; z = cz + (z - cz) * scI;
        pvx[p] *= 0.5; pvy[p] *= 0.5; pvz[p] *= 0.5;
      }
      if (ROCK(s, x, y, z)) {
        pAir[p] = 1; pvx[p] = pvy[p] = pvz[p] = 0;
        px[p] = (st_t)x; py[p] = (st_t)y; pz[p] = (st_t)z;
        continue;
      }
      double ciF = floor(x / dx), cjF = floor(y / dx), ckF = floor(z / dx);
      if (ciF >= 0 && cjF >= 0 && ckF >= 0 && ciF < nx && cjF < ny && ckF < nz &&
          type[((long)ckF * ny + (long)cjF) * nx + (long)ciF] == FLUID) {
        double exF = x - cx, eyF = y - cy, ezF = z - cz;
        double elF = sqrt(exF * exF + eyF * eyF + ezF * ezF); if (elF == 0) elF = 1e-9;
        double stepF = dx * 0.5;
        for (int mf = 0; mf < 12; mf++) {
          double qxI = x + exF / elF * stepF, qyI = y + eyF / elF * stepF, qzI = z + ezF / elF * stepF;
          double qi = floor(qxI / dx), qj = floor(qyI / dx), qk = floor(qzI / dx);
          if (qi < 0 || qj < 0 || qk < 0 || qi >= nx || qj >= ny || qk >= nz) break;
          if (type[((long)qk * ny + (long)qj) * nx + (long)qi] != FLUID) break;
          x = qxI; y = qyI; z = qzI;
        }
        pAir[p] = 1; pvx[p] = pvy[p] = pvz[p] = 0;
        s->pWx[p] = 0; s->pWy[p] = 0; s->pWz[p] = 0;
      }
      px[p] = (st_t)x; py[p] = (st_t)y; pz[p] = (st_t)z;
      continue;
    }
    if (fl[p] == 1 || fl[p] == 4) {                               /* ballistic, :1865-1976 */
      double gx = x - cx, gy = y - cy, gz = z - cz;
      double gr2 = gx * gx + gy * gy + gz * gz;
      double ga = g * oceanR * oceanR * dt / (gr2 * sqrt(gr2));
      pvx[p] = (st_t)(vx - gx * ga); pvy[p] = (st_t)(vy - gy * ga); pvz[p] = (st_t)(vz - gz * ga);
      double dr = 1 - 2.5 * dt; if (dr < 0) dr = 0;
      pvx[p] *= dr; pvy[p] *= dr; pvz[p] *= dr;
      double dsp = sqrt((double)pvx[p] * pvx[p] + (double)pvy[p] * pvy[p] + (double)pvz[p] * pvz[p]);
      if (dsp > maxSpeed) { double dsc = maxSpeed / dsp; pvx[p] *= dsc; pvy[p] *= dsc; pvz[p] *= dsc; }
      x += pvx[p] * dt; y += pvy[p] * dt; z += pvz[p] * dt;
      double bx = x - cx, by = y - cy, bz = z - cz;
      double br = sqrt(bx * bx + by * by + bz * bz); if (br == 0) br = 1e-9;
      double skyHi = oceanR + s->P.atmosphereH;
      if (br > skyHi) {
        double sc0 = skyHi / br;
        x = cx + bx * sc0; y = cy + by * sc0; z = cz + bz * sc0;
        double vr0 = ((double)pvx[p] * bx + (double)pvy[p] * by + (double)pvz[p] * bz) / br;
        if (vr0 > 0) {
          pvx[p] -= bx / br * vr0 * 1.15; pvy[p] -= by / br * vr0 * 1.15; pvz[p] -= bz / br * vr0 * 1.15;
        }
      } else if (br <= domHi) {
        int tries0 = 0;
        while (hasTerr && ROCK(s, x, y, z) && tries0 < 8) {
          double rW0 = sqrt((x - cx) * (x - cx) + (y - cy) * (y - cy) + (z - cz) * (z - cz));
          double stW0 = jmin(dx * 0.5, domHi - rW0);
          if (stW0 <= 1e-5) { tries0 = 8; break; }
          x += bx / br * stW0; y += by / br * stW0; z += bz / br * stW0;
          tries0++;
        }
        if (!hasTerr && br < coreLo) {
          double sc1 = coreLo / br;
          x = cx + bx * sc1; y = cy + by * sc1; z = cz + bz * sc1;
          tries0 = 1;
        }
        if (tries0 > 0) {
          if (hasTerr) {
            double exS = x - cx, eyS = y - cy, ezS = z - cz;
            double erS = sqrt(exS * exS + eyS * eyS + ezS * ezS); if (erS == 0) erS = 1e-9;
            double wantS = TRAD(s, x, y, z) + dx * 0.06;
            if (erS > wantS) { x = cx + exS / erS * wantS; y = cy + eyS / erS * wantS; z = cz + ezS / erS * wantS; }
            int kS = 0;
            while (ROCK(s, x, y, z) && kS < 4) {
              x += exS / erS * dx * 0.5; y += eyS / erS * dx * 0.5; z += ezS / erS * dx * 0.5;
              kS++;
            }
          }
          double vr1 = ((double)pvx[p] * bx + (double)pvy[p] * by + (double)pvz[p] * bz) / br;
          pvx[p] -= bx / br * vr1; pvy[p] -= by / br * vr1; pvz[p] -= bz / br * vr1;
          pvx[p] *= 0.3; pvy[p] *= 0.3; pvz[p] *= 0.3;
          fl[p] = 0;
        }
      }
      px[p] = (st_t)x; py[p] = (st_t)y; pz[p] = (st_t)z;
      int ci = jfloor_clamp(x / dx, 0, nx - 1), cj = jfloor_clamp(y / dx, 0, ny - 1), ck = jfloor_clamp(z / dx, 0, nz - 1);
      long c = ((long)ck * ny + cj) * nx + ci;
      if (type[c] == FLUID) {
        pvx[p] *= 0.45; pvy[p] *= 0.45; pvz[p] *= 0.45;
        if (pvy[p] > 0.5) pvy[p] = 0.5f;
        pcool[p] = 2;
        fl[p] = 0;
      }
      continue;
    }
    if (fl[p] == 2 || fl[p] == 3) {                               /* atmosphere, :1978-2174 */
      double Tv = s->pT[p];
      pAir[p] += dt;
      double vEx = x - cx, vEy = y - cy, vEz = z - cz;
      double vEr = sqrt(vEx * vEx + vEy * vEy + vEz * vEz); if (vEr == 0) vEr = 1e-9;
      double ux = vEx / vEr, uy = vEy / vEr, uz = vEz / vEr;
      double exposure = ux * windSX + uy * windSY + uz * windSZ;
      double jet = jmin(oceanR * 0.58, maxSpeed * 0.45);
      double returnFlow = jmin(oceanR * 0.32, maxSpeed * 0.25);
      double vr = vx * ux + vy * uy + vz * uz;
      double radial = -s->P.gravity * 0.06;
      double wx = -uz * jet - (windSX - exposure * ux) * returnFlow;
      double wy = -(windSY - exposure * uy) * returnFlow;
      double wz = ux * jet - (windSZ - exposure * uz) * returnFlow;
      double relax = jmin(1, dt * 1.3);
      pvx[p] = (st_t)(vx + (wx - (vx - vr * ux)) * relax + ux * radial * dt);
      pvy[p] = (st_t)(vy + (wy - (vy - vr * uy)) * relax + uy * radial * dt);
      pvz[p] = (st_t)(vz + (wz - (vz - vr * uz)) * relax + uz * radial * dt);
      double svv = (double)pvx[p] * pvx[p] + (double)pvy[p] * pvy[p] + (double)pvz[p] * pvz[p];
      if (svv > maxSpeed * maxSpeed) {
        double svs = maxSpeed / sqrt(svv);
        pvx[p] *= svs; pvy[p] *= svs; pvz[p] *= svs;
      }
      x += pvx[p] * dt; y += pvy[p] * dt; z += pvz[p] * dt;
      int backToSea;
      double vCx = x - cx, vCy = y - cy, vCz = z - cz;
      double vCr = sqrt(vCx * vCx + vCy * vCy + vCz * vCz); if (vCr == 0) vCr = 1e-9;
      double ceilR = oceanR + s->P.atmosphereH - 1e-3 * dx;
      if (hasTerr) { double RtE = TRAD(s, x, y, z); if (RtE + 0.02 > ceilR) ceilR = RtE + 0.02; }
      if (vCr > ceilR) {
        double scE = ceilR / vCr;
        x = cx + vCx * scE; y = cy + vCy * scE; z = cz + vCz * scE;
        double vrE = ((double)pvx[p] * vCx + (double)pvy[p] * vCy + (double)pvz[p] * vCz) / vCr;
        if (vrE > 0) { pvx[p] -= vCx / vCr * vrE * 2; pvy[p] -= vCy / vCr * vrE * 2; pvz[p] -= vCz / vCr * vrE * 2; }
      }
      double vrC2 = ((double)pvx[p] * vCx + (double)pvy[p] * vCy + (double)pvz[p] * vCz) / vCr;
      if (vrC2 > 0 && vCr > oceanR) {
        double hh = (vCr - oceanR) / (s->P.atmosphereH > 1e-4 ? s->P.atmosphereH : 1e-4);
        if (hh > 1) hh = 1;
        double prf = s->P.ceilReflect == 1 ? hh * hh : s->P.ceilReflect == 2 ? (exp(3 * hh) - 1) * 0.0523957 : hh;
        if (prf > 0) {
          s->S.cfS = lcg(s->S.cfS);
          if (s->S.cfS / 4294967296.0 < prf * dt * 4) {
            pvx[p] -= vCx / vCr * vrC2 * 2; pvy[p] -= vCy / vCr * vrC2 * 2; pvz[p] -= vCz / vCr * vrC2 * 2;
          }
        }
      }
      double fCx = x - cx, fCy = y - cy, fCz = z - cz;
      double fCr = sqrt(fCx * fCx + fCy * fCy + fCz * fCz); if (fCr == 0) fCr = 1e-9;
      double floorR = oceanR + 0.15 * dx;
      if (fCr < floorR) {
        double vrF = ((double)pvx[p] * fCx + (double)pvy[p] * fCy + (double)pvz[p] * fCz) / fCr;
        if (vrF < 0) {
          s->S.bfS = lcg(s->S.bfS);
          if (s->S.bfS / 4294967296.0 < 0.07) {
            double scF = floorR / fCr;
            x = cx + fCx * scF; y = cy + fCy * scF; z = cz + fCz * scF;
            pvx[p] -= fCx / fCr * vrF * 2; pvy[p] -= fCy / fCr * vrF * 2; pvz[p] -= fCz / fCr * vrF * 2;
          } else {
            double scB = (floorR + 0.02 * dx) / fCr;
            x = cx + fCx * scB; y = cy + fCy * scB; z = cz + fCz * scB;
            pvx[p] -= fCx / fCr * vrF * 2; pvy[p] -= fCy / fCr * vrF * 2; pvz[p] -= fCz / fCr * vrF * 2;
          }
        }
      }
      int triesE = 0;
      double rNow3 = sqrt((x - cx) * (x - cx) + (y - cy) * (y - cy) + (z - cz) * (z - cz));
      while (hasTerr && rNow3 < s->domainR && ROCK(s, x, y, z) && triesE < 8) {
        double rW3 = sqrt((x - cx) * (x - cx) + (y - cy) * (y - cy) + (z - cz) * (z - cz));
        double stW3 = jmin(dx * 0.5, domHi - rW3);
        if (stW3 <= 1e-5) break;
        x += vCx / vCr * stW3; y += vCy / vCr * stW3; z += vCz / vCr * stW3;
        triesE++;
      }
      if (triesE > 0) {
        double vrT = ((double)pvx[p] * vCx + (double)pvy[p] * vCy + (double)pvz[p] * vCz) / vCr;
        if (vrT < 0) {
          double bT = 1.5 * vrT / vCr;
          pvx[p] -= vCx * bT; pvy[p] -= vCy * bT; pvz[p] -= vCz * bT;
        }
        pvx[p] *= 0.92; pvy[p] *= 0.92; pvz[p] *= 0.92;
      }
      int ciV = jfloor_clamp(x / dx, 0, nx - 1), cjV = jfloor_clamp(y / dx, 0, ny - 1), ckV = jfloor_clamp(z / dx, 0, nz - 1);
      backToSea = type[((long)ckV * ny + cjV) * nx + ciV] == FLUID;
      if (backToSea) {
        double bx2 = x - cx, by2 = y - cy, bz2 = z - cz;
        double br2 = sqrt(bx2 * bx2 + by2 * by2 + bz2 * bz2); if (br2 == 0) br2 = 1e-9;
        if (br2 > oceanR + 0.15 * dx) backToSea = 0;
        else if (((double)pvx[p] * bx2 + (double)pvy[p] * by2 + (double)pvz[p] * bz2) / br2 > 0.02) backToSea = 0;
      }
      px[p] = (st_t)x; py[p] = (st_t)y; pz[p] = (st_t)z;
      if (backToSea) {
        pvx[p] = 0; pvy[p] = 0; pvz[p] = 0; pAir[p] = 0; fl[p] = 0;
      } else if (fl[p] == 2 && ((Tv <= rainTe && pAir[p] >= s->P.rainLiftAge) || pAir[p] > 40)) {
        pvx[p] = 0; pvy[p] = 0; pvz[p] = 0; pAir[p] = 0; fl[p] = 4;
      }
      continue;
    }
    /* grid-coupled fluid, :2176-2290 */
    double t0[3];
    if (s->gridSampleValid) { t0[0] = s->advU[p]; t0[1] = s->advV[p]; t0[2] = s->advW[p]; }
    else sample_vel3(s, x, y, z, t0);
    double sp2 = t0[0] * t0[0] + t0[1] * t0[1] + t0[2] * t0[2];
    double v2x = t0[0], v2y = t0[1], v2z = t0[2];
    if (sp2 > 0.25) {
      double mx = jclampd(x + 0.5 * dt * t0[0], xLo, xHi);
      double my = jclampd(y + 0.5 * dt * t0[1], yLo, yHi);
      double mz = jclampd(z + 0.5 * dt * t0[2], zLo, zHi);
      double t2[3]; sample_vel3(s, mx, my, mz, t2);
      v2x = t2[0]; v2y = t2[1]; v2z = t2[2];
    }
    sp2 = v2x * v2x + v2y * v2y + v2z * v2z;
    if (sp2 > maxSpeed * maxSpeed) {
      double sc = maxSpeed / sqrt(sp2);
      v2x *= sc; v2y *= sc; v2z *= sc;
      pvx[p] *= sc; pvy[p] *= sc; pvz[p] *= sc;
    }
    x += v2x * dt; y += v2y * dt; z += v2z * dt;
    double nx2 = x - cx, ny2 = y - cy, nz2 = z - cz;
    double nr = sqrt(nx2 * nx2 + ny2 * ny2 + nz2 * nz2); if (nr == 0) nr = 1e-9;
    if (nr > domHi) {
      double sc2 = domHi / nr;
      x = cx + nx2 * sc2; y = cy + ny2 * sc2; z = cz + nz2 * sc2;
      pvy[p] = (st_t)(-fabs((double)pvy[p]) * 0.1 - 0.3);
      fl[p] = 1;
    }
    if (nr < domHi) {
      int tries = 0;
      while (hasTerr && ROCK(s, x, y, z) && tries < 8) {
        double rW2 = sqrt((x - cx) * (x - cx) + (y - cy) * (y - cy) + (z - cz) * (z - cz));
        double stW2 = jmin(dx * 0.5, domHi - rW2);
        if (stW2 <= 1e-5) { tries = 8; break; }
        x += nx2 / nr * stW2; y += ny2 / nr * stW2; z += nz2 / nr * stW2;
        tries++;
      }
      if (tries > 0) {
        if (hasTerr) {
          double exS2 = x - cx, eyS2 = y - cy, ezS2 = z - cz;
          double erS2 = sqrt(exS2 * exS2 + eyS2 * eyS2 + ezS2 * ezS2); if (erS2 == 0) erS2 = 1e-9;
          double wantS2 = TRAD(s, x, y, z) + dx * 0.06;
          if (erS2 > wantS2) { x = cx + exS2 / erS2 * wantS2; y = cy + eyS2 / erS2 * wantS2; z = cz + ezS2 / erS2 * wantS2; }
          int kS2 = 0;
          while (ROCK(s, x, y, z) && kS2 < 4) {
            x += exS2 / erS2 * dx * 0.5; y += eyS2 / erS2 * dx * 0.5; z += ezS2 / erS2 * dx * 0.5;
            kS2++;
          }
        }
        double vr2 = ((double)pvx[p] * nx2 + (double)pvy[p] * ny2 + (double)pvz[p] * nz2) / nr;
        if (vr2 < 0) { pvx[p] -= nx2 / nr * vr2; pvy[p] -= ny2 / nr * vr2; pvz[p] -= nz2 / nr * vr2; }
      }
      if (hasTerr && (tries > 0 || ROCK(s, x - nx2 / nr * dx, y - ny2 / nr * dx, z - nz2 / nr * dx))) {
        double fr0 = 1 - 0.6 * dt; if (fr0 < 0) fr0 = 0;
        pvx[p] *= fr0; pvy[p] *= fr0; pvz[p] *= fr0;
      }
    }
    double sx = x - cx, sy = y - cy, sz = z - cz;
    double sr = sqrt(sx * sx + sy * sy + sz * sz); if (sr == 0) sr = 1e-9;
    double vrad = ((double)pvx[p] * sx + (double)pvy[p] * sy + (double)pvz[p] * sz) / sr;
    double da = 1.0 * dt; if (da > 0.5) da = 0.5;
    pvx[p] -= sx / sr * vrad * da; pvy[p] -= sy / sr * vrad * da; pvz[p] -= sz / sr * vrad * da;
    double dg = 1 - 0.42 * dt; if (dg < 0) dg = 0;
    pvx[p] *= dg; pvy[p] *= dg; pvz[p] *= dg;
    px[p] = (st_t)x; py[p] = (st_t)y; pz[p] = (st_t)z;
  }
  s->gridSampleValid = 0;
}

/* ------------------------------------------------------------ balls
 * addBall (js/solver.js:3910-3912), _pushBallsChunk (:1009-1026),
 * _ballVsTerrain (:2299-2342) and _updateBalls (:2344-2564), sphere world. */
int or_add_ball(or_solver* s, double x, double y, double z, double r, double rho) {
  if (s->nBalls >= OR_MAX_BALLS) return -1;
  double* b = s->balls[s->nBalls++];
  b[BX] = x; b[BY] = y; b[BZ] = z; b[BVX] = b[BVY] = b[BVZ] = 0; b[BR] = r; b[BRHO] = rho; b[BSUB] = 0;
  return s->nBalls;
}
int or_get_balls(or_solver* s, double* out, int max) {
  for (int n = 0; n < s->nBalls && n < max; n++) memcpy(out + 9 * n, s->balls[n], sizeof(double) * 9);
  return s->nBalls;
}
int or_set_balls(or_solver* s, const double* in, int count) {
  if (count < 0 || count > OR_MAX_BALLS) return -1;
  for (int n = 0; n < count; n++) memcpy(s->balls[n], in + 9 * n, sizeof(double) * 9);
  s->nBalls = count;
  return count;
}
void or_push_balls(or_solver* s) {
  int nP = s->S.nP;
  for (int n = 0; n < s->nBalls; n++) {
    const double* b = s->balls[n];
    double rr = b[BR] + 0.002;
    for (int p = 0; p < nP; p++) {
      double ex = s->px[p] - b[BX], ey = s->py[p] - b[BY], ez = s->pz[p] - b[BZ];
      double d2 = ex * ex + ey * ey + ez * ez;
      if (d2 < rr * rr) {
        double d = sqrt(d2); if (!(d != 0)) d = 1e-9;
        double inv = 1 / d, nxn = ex * inv, nyn = ey * inv, nzn = ez * inv;
        s->px[p] = (st_t)(b[BX] + nxn * rr); s->py[p] = (st_t)(b[BY] + nyn * rr); s->pz[p] = (st_t)(b[BZ] + nzn * rr);
        double rvx = s->pvx[p] - b[BVX], rvy = s->pvy[p] - b[BVY], rvz = s->pvz[p] - b[BVZ];
        double vn = rvx * nxn + rvy * nyn + rvz * nzn;
        if (vn < 0) {
          s->pvx[p] = (st_t)(s->pvx[p] - nxn * vn); s->pvy[p] = (st_t)(s->pvy[p] - nyn * vn);
          s->pvz[p] = (st_t)(s->pvz[p] - nzn * vn);
        }
      }
    }
  }
}
static void ball_vs_terrain(or_solver* s, double* b) {
  int n = s->tn; double dv = s->tdv; const uint8_t* solid = s->tsolid;
  int i0 = jtrunc((b[BX] - b[BR]) / dv), i1 = jtrunc((b[BX] + b[BR]) / dv);
  int j0 = jtrunc((b[BY] - b[BR]) / dv), j1 = jtrunc((b[BY] + b[BR]) / dv);
  int k0 = jtrunc((b[BZ] - b[BR]) / dv), k1 = jtrunc((b[BZ] + b[BR]) / dv);
  if (i0 < 0) i0 = 0;
  if (j0 < 0) j0 = 0;
  if (k0 < 0) k0 = 0;
  if (i1 > n - 1) i1 = n - 1;
  if (j1 > n - 1) j1 = n - 1;
  if (k1 > n - 1) k1 = n - 1;
  double bestPen = 0, bpx = 0, bpy = 0, bpz = 0;
  for (int k = k0; k <= k1; k++) for (int j = j0; j <= j1; j++) {
    long rowB = ((long)k * n + j) * n;
    for (int i = i0; i <= i1; i++) {
      if (!solid[rowB + i]) continue;
      double qx = b[BX], qy = b[BY], qz = b[BZ];
      double vx0 = i * dv, vy0 = j * dv, vz0 = k * dv;
      if (qx < vx0) qx = vx0; else if (qx > vx0 + dv) qx = vx0 + dv;
      if (qy < vy0) qy = vy0; else if (qy > vy0 + dv) qy = vy0 + dv;
      if (qz < vz0) qz = vz0; else if (qz > vz0 + dv) qz = vz0 + dv;
      double ddx = b[BX] - qx, ddy = b[BY] - qy, ddz = b[BZ] - qz;
      double dd = sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
      double pen = b[BR] - dd;
      if (pen > bestPen) {
        if (dd > 1e-6) { bestPen = pen; bpx = ddx / dd; bpy = ddy / dd; bpz = ddz / dd; }
        else {
          double rx = b[BX] - s->cx, ry = b[BY] - s->cy, rz = b[BZ] - s->cz;
          double rl = sqrt(rx * rx + ry * ry + rz * rz); if (!(rl != 0)) rl = 1e-9;
          bestPen = pen; bpx = rx / rl; bpy = ry / rl; bpz = rz / rl;
        }
      }
    }
  }
  if (bestPen > 0) {
    b[BX] += bpx * (bestPen + 0.002); b[BY] += bpy * (bestPen + 0.002); b[BZ] += bpz * (bestPen + 0.002);
    double vn = b[BVX] * bpx + b[BVY] * bpy + b[BVZ] * bpz;
    if (vn < 0) {
      b[BVX] -= bpx * vn; b[BVY] -= bpy * vn; b[BVZ] -= bpz * vn;
      b[BVX] *= 0.985; b[BVY] *= 0.985; b[BVZ] *= 0.985;
    }
  }
}
void or_update_balls(or_solver* s, double dt) {
  const double rhoF = 1000, Cd = 0.5, PI = 3.141592653589793;
  int nb = s->nBalls, nP = s->S.nP;
  enum { HIST = 24 };
  if (nb > 0) {
    double hLo = s->S.coreR, hSpan = (s->S.oceanR - s->S.coreR) * 1.5;
    float hist[OR_MAX_BALLS * HIST]; int32_t histC[OR_MAX_BALLS];
    memset(hist, 0, sizeof(hist)); memset(histC, 0, sizeof(histC));
    for (int p = 0; p < nP; p++) {
      if (s->pflag[p] != 0) continue;
      double ppx = s->px[p], ppy = s->py[p], ppz = s->pz[p];
      double ldx = ppx - s->cx, ldy = ppy - s->cy, ldz = ppz - s->cz;
      double level = sqrt(ldx * ldx + ldy * ldy + ldz * ldz);
      for (int q = 0; q < nb; q++) {
        const double* bb = s->balls[q];
        double bdx = ppx - bb[BX], bdy = ppy - bb[BY], bdz = ppz - bb[BZ];
        double dh2 = bdx * bdx + bdy * bdy + bdz * bdz;
        double r1 = 2.2 * bb[BR], r2 = 3.2 * bb[BR];
        if (dh2 < r1 * r1 || dh2 > r2 * r2) continue;
        double bf = floor(((level - hLo) / hSpan) * HIST);
        histC[q]++;
        if (bf != bf) continue;                 /* NaN bucket: the reference's store is a no-op */
        int bucket = bf < 0 ? 0 : (bf >= HIST ? HIST - 1 : (int)bf);
        hist[q * HIST + bucket]++;
      }
    }
    for (int q = 0; q < nb; q++) {
      int total = histC[q]; double wl = -INFINITY;
      if (total > 20) {
        double acc = 0, target = total * 0.10;
        for (int bkt = HIST - 1; bkt >= 0; bkt--) {
          acc += hist[q * HIST + bkt];
          if (acc >= target) { wl = hLo + (bkt + 0.5) / HIST * hSpan; break; }
        }
        if (wl == -INFINITY || total < 140) wl = s->S.oceanR;
        double wlMax = s->S.oceanR + (s->S.oceanR - s->S.coreR) * 0.3;
        if (wl > wlMax) wl = wlMax;
        if (wl < s->S.coreR) wl = s->S.coreR;
      } else {
        wl = s->S.oceanR;
      }
      s->surfY[q] = (float)wl;
    }
  }
  double g = s->P.gravity;
  for (int n = 0; n < nb; n++) {
    double* b = s->balls[n];
    double m = b[BRHO] * 4 / 3 * PI * b[BR] * b[BR] * b[BR];
    double area = PI * b[BR] * b[BR];
    double surf = s->surfY[n];
    double ex0 = b[BX] - s->cx, ey0 = b[BY] - s->cy, ez0 = b[BZ] - s->cz;
    double bR = sqrt(ex0 * ex0 + ey0 * ey0 + ez0 * ez0);
    double inner = bR - b[BR], h = surf - inner;
    if (!(h > 0)) h = 0;
    if (h > 2 * b[BR]) h = 2 * b[BR];
    double Vs = PI * h * h * (3 * b[BR] - h) / 3;
    b[BSUB] = Vs / (4.0 / 3 * PI * b[BR] * b[BR] * b[BR]);
    double upx = 0, upy = 1, upz = 0, gEff = g;
    if (bR > 1e-6) {
      upx = (b[BX] - s->cx) / bR; upy = (b[BY] - s->cy) / bR; upz = (b[BZ] - s->cz) / bR;
      gEff = g * (s->S.oceanR * s->S.oceanR) / (bR * bR);
    }
    double Fb = (rhoF * Vs - m) * gEff;
    double tmp[3];
    sample_vel3(s, b[BX], b[BY], b[BZ], tmp);
    double rvx = b[BVX] - tmp[0], rvy = b[BVY] - tmp[1], rvz = b[BVZ] - tmp[2];
    double vr = sqrt(rvx * rvx + rvy * rvy + rvz * rvz);
    double kd = 0.5 * rhoF * Cd * area * vr;
    double Fx = -kd * rvx + upx * Fb, Fz = -kd * rvz + upz * Fb, Fyd = -kd * rvy + upy * Fb;
    double fdx = Fx - upx * Fb, fdy = Fyd - upy * Fb, fdz = Fz - upz * Fb;
    double fdm = sqrt(fdx * fdx + fdy * fdy + fdz * fdz);
    double fdmMax = 0.8 * m * g;
    if (fdm > fdmMax) {
      double fdc = fdmMax / fdm;
      Fx = upx * Fb + fdx * fdc; Fyd = upy * Fb + fdy * fdc; Fz = upz * Fb + fdz * fdc;
    }
    double mEff = m + 0.5 * rhoF * Vs;
    b[BVX] += (Fx / mEff) * dt;
    b[BVZ] += (Fz / mEff) * dt;
    b[BVY] += (Fyd / mEff) * dt;
    b[BVX] *= 0.999; b[BVY] *= 0.999; b[BVZ] *= 0.999;
    const double bvmax = 4;
    if (b[BVX] > bvmax) b[BVX] = bvmax; else if (b[BVX] < -bvmax) b[BVX] = -bvmax;
    if (b[BVZ] > bvmax) b[BVZ] = bvmax; else if (b[BVZ] < -bvmax) b[BVZ] = -bvmax;
    if (b[BVY] > bvmax) b[BVY] = bvmax; else if (b[BVY] < -bvmax) b[BVY] = -bvmax;
    b[BX] += b[BVX] * dt; b[BY] += b[BVY] * dt; b[BZ] += b[BVZ] * dt;
    if (s->hasTerr) {
      ball_vs_terrain(s, b);
    } else {
      double cbx = b[BX] - s->cx, cby = b[BY] - s->cy, cbz = b[BZ] - s->cz;
      double cbr = sqrt(cbx * cbx + cby * cby + cbz * cbz); if (!(cbr != 0)) cbr = 1e-9;
      if (cbr < s->S.coreR + b[BR]) {
        double rnx0 = cbx / cbr, rny0 = cby / cbr, rnz0 = cbz / cbr, rr0 = s->S.coreR + b[BR];
        b[BX] = s->cx + rnx0 * rr0; b[BY] = s->cy + rny0 * rr0; b[BZ] = s->cz + rnz0 * rr0;
        double vn0 = b[BVX] * rnx0 + b[BVY] * rny0 + b[BVZ] * rnz0;
        if (vn0 < 0) {
          b[BVX] -= rnx0 * vn0 * 1.3; b[BVY] -= rny0 * vn0 * 1.3; b[BVZ] -= rnz0 * vn0 * 1.3;
          b[BVX] *= 0.98; b[BVY] *= 0.98; b[BVZ] *= 0.98;
        }
      }
    }
    double sbx = b[BX] - s->cx, sby = b[BY] - s->cy, sbz = b[BZ] - s->cz;
    double sbr = sqrt(sbx * sbx + sby * sby + sbz * sbz); if (!(sbr != 0)) sbr = 1e-9;
    double rnx = sbx / sbr, rny = sby / sbr, rnz = sbz / sbr;
    if (sbr > s->domainR - b[BR]) {
      double rr1 = s->domainR - b[BR];
      b[BX] = s->cx + rnx * rr1; b[BY] = s->cy + rny * rr1; b[BZ] = s->cz + rnz * rr1;
      double vn1 = b[BVX] * rnx + b[BVY] * rny + b[BVZ] * rnz;
      if (vn1 > 0) { b[BVX] -= rnx * vn1 * 1.3; b[BVY] -= rny * vn1 * 1.3; b[BVZ] -= rnz * vn1 * 1.3; }
    }
  }
  for (int a = 0; a < nb; a++) for (int c = a + 1; c < nb; c++) {
    double *A = s->balls[a], *B = s->balls[c];
    double ex = B[BX] - A[BX], ey = B[BY] - A[BY], ez = B[BZ] - A[BZ];
    double d2 = ex * ex + ey * ey + ez * ez, rSum = A[BR] + B[BR];
    if (d2 > rSum * rSum || d2 < 1e-12) continue;
    double d = sqrt(d2), nxn = ex / d, nyn = ey / d, nzn = ez / d;
    double overlap = rSum - d;
    double mA = A[BRHO] * A[BR] * A[BR] * A[BR], mB = B[BRHO] * B[BR] * B[BR] * B[BR];
    double tA = mB / (mA + mB), tB = mA / (mA + mB);
    A[BX] -= nxn * overlap * tA; A[BY] -= nyn * overlap * tA; A[BZ] -= nzn * overlap * tA;
    B[BX] += nxn * overlap * tB; B[BY] += nyn * overlap * tB; B[BZ] += nzn * overlap * tB;
    double rvn = (B[BVX] - A[BVX]) * nxn + (B[BVY] - A[BVY]) * nyn + (B[BVZ] - A[BVZ]) * nzn;
    if (rvn < 0) {
      double jimp = -(1 + 0.3) * rvn / (1 / mA + 1 / mB);
      A[BVX] -= nxn * jimp / mA; A[BVY] -= nyn * jimp / mA; A[BVZ] -= nzn * jimp / mA;
      B[BVX] += nxn * jimp / mB; B[BVY] += nyn * jimp / mB; B[BVZ] += nzn * jimp / mB;
    }
  }
}

/* ------------------------------------------------------------ substep
 * _substep, js/solver.js:2568-2624 (sphere mode) */
void or_substep(or_solver* s, double dt) {
  or_clear_faces(s);
  or_rasterize_static(s);
  or_mark_fluid(s);
  if (s->nBalls) or_push_balls(s);
  or_p2g(s);
  or_apply_bc(s);
  or_snapshot_old(s);
  or_viscosity(s, dt);
  or_planet_gravity(s, dt);
  or_apply_bc(s);
  or_pressure_solve(s);
  or_project(s);
  if (s->P.vorticity > 0) or_vorticity(s, dt);
  s->S.umax = or_clamp_um(s);
  or_extrapolate(s);
  or_g2p(s, dt);
  or_advect(s, dt);
  if (s->nBalls) or_push_balls(s);
  s->gridSampleValid = 0;
  if (s->nBalls) or_update_balls(s, dt);
  s->S.dtLast = dt;
}

/* ------------------------------------------------------------ currents
 * Subsurface currents, js/solver.js:3624-3782: nine sum-of-sines waves of a
 * vector potential (seeded LCG, _buildCurrWaves :3634-3656), its analytic curl
 * sampled on a lattice of stride 4 cells (float storage, :3682-3722), and a
 * capped relaxation of deep fluid particles toward the tangential part of the
 * trilinearly sampled current (:3726-3782). */
typedef struct { double kx, ky, kz, A, ph; } cwave_t;
static void curr_waves(cwave_t w[3][3], double drift[3]) {
  double seed = 1234567;
  const double K[3] = { 1.5, 4.0, 9.0 }, amp[3] = { 0.10, 0.085, 0.05 }, dr[3] = { 0.021, 0.05, 0.11 };
  for (int o = 0; o < 3; o++) {
    for (int c = 0; c < 3; c++) {
      double r3[3];
      for (int q = 0; q < 3; q++) { seed = fmod(seed * 1664525 + 1013904223, 4294967296.0); r3[q] = seed / 4294967296.0 * 2 - 1; }
      double L = sqrt(r3[0] * r3[0] + r3[1] * r3[1] + r3[2] * r3[2]); if (L == 0) L = 1;
      w[o][c].kx = r3[0] / L * K[o]; w[o][c].ky = r3[1] / L * K[o]; w[o][c].kz = r3[2] / L * K[o];
      w[o][c].A = amp[o] / K[o];
      seed = fmod(seed * 1664525 + 1013904223, 4294967296.0);
      w[o][c].ph = seed / 4294967296.0 * 6.283;
    }
    drift[o] = dr[o];
  }
}
void or_update_currents(or_solver* s, double dt) {
  double strength = s->P.currents, shell = s->S.oceanR - s->S.coreR;
  if (!(strength > 0) || !(shell > 0)) return;
  const int stride = 4;
  int gnx = s->nx / stride + 2, gny = s->ny / stride + 2, gnz = s->nz / stride + 2;
  long gN = (long)gnx * gny * gnz;
  float* cfx = (float*)malloc(sizeof(float) * gN); float* cfy = (float*)malloc(sizeof(float) * gN);
  float* cfz = (float*)malloc(sizeof(float) * gN);
  cwave_t w[3][3]; double drift[3];
  curr_waves(w, drift);
  double sx = s->dx * stride, t = s->S.simTime, ampl = strength * 2;
  for (int kk = 0; kk < gnz; kk++) for (int jj = 0; jj < gny; jj++) for (int ii = 0; ii < gnx; ii++) {
    double wx2 = ii * sx, wy2 = jj * sx, wz2 = kk * sx, ux = 0, uy = 0, uz = 0;
    for (int o = 0; o < 3; o++) {
      double dph = drift[o] * t;
      double thx = w[o][0].kx * wx2 + w[o][0].ky * wy2 + w[o][0].kz * wz2 + dph + w[o][0].ph;
      double thy = w[o][1].kx * wx2 + w[o][1].ky * wy2 + w[o][1].kz * wz2 + dph + w[o][1].ph;
      double thz = w[o][2].kx * wx2 + w[o][2].ky * wy2 + w[o][2].kz * wz2 + dph + w[o][2].ph;
      ux += w[o][2].A * w[o][2].ky * cos(thz) - w[o][1].A * w[o][1].kz * cos(thy);
      uy += w[o][0].A * w[o][0].kz * cos(thx) - w[o][2].A * w[o][2].kx * cos(thz);
      uz += w[o][1].A * w[o][1].kx * cos(thy) - w[o][0].A * w[o][0].ky * cos(thx);
    }
    long gi = ((long)kk * gny + jj) * gnx + ii;
    cfx[gi] = (float)(ux * ampl); cfy[gi] = (float)(uy * ampl); cfz[gi] = (float)(uz * ampl);
  }
  double relax = 2.2 * dt; if (relax > 0.35) relax = 0.35;
  const double dvCap = 0.15, invS = 1 / (s->dx * stride);
  long gxy = (long)gnx * gny;
  int kmax = s->nz / stride;
  for (int p = 0; p < s->S.nP; p++) {
    if (s->pflag[p] != 0) continue;
    double rx = s->px[p] - s->cx, ry = s->py[p] - s->cy, rz = s->pz[p] - s->cz;
    double rl = sqrt(rx * rx + ry * ry + rz * rz); if (rl == 0) rl = 1e-9;
    double dpt = (s->S.oceanR - rl) / shell;
    double wgt = (dpt - 0.06) * 4.0;
    if (wgt <= 0) continue;
    if (wgt > 1) wgt = 1;
    double qa = s->px[p] * invS, qb = s->py[p] * invS, qc = s->pz[p] * invS;
    int i0 = jtrunc(qa), j0 = jtrunc(qb), k0 = jtrunc(qc);
    if (i0 > gnx - 2) i0 = gnx - 2; else if (i0 < 0) i0 = 0;
    if (j0 > gny - 2) j0 = gny - 2; else if (j0 < 0) j0 = 0;
    if (k0 > kmax) k0 = kmax; else if (k0 < 0) k0 = 0;
    double ta = qa - i0; if (ta > 1) ta = 1; else if (ta < 0) ta = 0;
    double tb = qb - j0; if (tb > 1) tb = 1; else if (tb < 0) tb = 0;
    double tc = qc - k0; if (tc > 1) tc = 1; else if (tc < 0) tc = 0;
    long g = ((long)k0 * gny + j0) * gnx + i0;
    double a0 = 1 - ta, a1 = ta, b0 = 1 - tb, b1 = tb, c0 = 1 - tc, c1 = tc;
#define CSAMP(f) ((f[g] * a0 + f[g + 1] * a1) * b0 * c0 + (f[g + gnx] * a0 + f[g + gnx + 1] * a1) * b1 * c0 + \
                  (f[g + gxy] * a0 + f[g + gxy + 1] * a1) * b0 * c1 + (f[g + gxy + gnx] * a0 + f[g + gxy + gnx + 1] * a1) * b1 * c1)
    double Ux = CSAMP(cfx), Uy = CSAMP(cfy), Uz = CSAMP(cfz);
#undef CSAMP
    double ir = 1 / rl;
    double Ur = (Ux * rx + Uy * ry + Uz * rz) * ir;
    double Tx = (Ux - rx * ir * Ur) * wgt, Ty = (Uy - ry * ir * Ur) * wgt, Tz = (Uz - rz * ir * Ur) * wgt;
    double vr = ((double)s->pvx[p] * rx + (double)s->pvy[p] * ry + (double)s->pvz[p] * rz) * ir;
    double vx = s->pvx[p] - rx * ir * vr, vy = s->pvy[p] - ry * ir * vr, vz = s->pvz[p] - rz * ir * vr;
    double ex = relax * (Tx - vx), ey = relax * (Ty - vy), ez = relax * (Tz - vz);
    double e2 = ex * ex + ey * ey + ez * ez;
    if (e2 > dvCap * dvCap) { double es = dvCap / sqrt(e2); ex *= es; ey *= es; ez *= es; }
    s->pvx[p] = (st_t)(s->pvx[p] + ex); s->pvy[p] = (st_t)(s->pvy[p] + ey); s->pvz[p] = (st_t)(s->pvz[p] + ez);
  }
  free(cfx); free(cfy); free(cfz);
}

/* _stepSync, js/solver.js:2670-2700. thermalOn=0 skips the atmospheric
 * cycle (heat tick, evaporation, vapour collisions, phases, ice contacts). */
void or_step(or_solver* s, double dtFrame) {
  s->S.simTime += dtFrame;
  if (s->P.thermalOn && s->S.capacity > 1) {
    s->S.heatAcc = s->S.heatAcc + dtFrame;
    if (s->S.heatAcc >= 1.0 / 25) {
      double dtTick = jmin(s->S.heatAcc, 1.0 / 12);
      or_update_heat(s, dtTick);
      if (s->P.sunActivity > 0) or_update_evaporation(s, dtTick);
      if (s->P.currents > 0) or_update_currents(s, dtTick);
      s->S.heatAcc = 0;
    }
  }
  double remaining = dtFrame; int guard = 0, nSub = 0;
  double base = dtFrame / jmax(1, s->P.substeps);
  while (remaining > 1e-6 && guard < 10) {
    double dt = jmin(jmin(base, (s->P.cfl * s->dx) / jmax(s->S.umax, 0.08)), 1.0 / 100);
    if (dt < 1e-5) dt = 1e-5;
    or_substep(s, dt);
    remaining -= dt; guard++; nSub++;
  }
  s->S.substepsLast = nSub;
  if (s->P.thermalOn) {
    or_vapor_collisions(s);
    or_update_phase(s, dtFrame);
    or_ice_contacts(s);
  }
  or_push_surface(s);
}

/* ------------------------------------------------------------ thermal
 * _updateHeat and helpers, js/solver.js:2715-2994 */
void or_update_heat(or_solver* s, double dt) {
  int nP = s->S.nP, nx = s->nx, ny = s->ny, nz = s->nz, N = s->nCells, p, c;
  if (nP < 1) return;
  double dx = s->dx;
  s->heatDt = dt;
  s->heatAlpha = jmin(s->P.heatK * dt * 0.15, 0.14);
  /* bins: count + prefix (:2731-2755), fill in index order (:2758-2770) */
  if (s->hOrdCap < nP) { free(s->hOrd); s->hOrd = xcalloc((size_t)nP * 2, sizeof(int32_t)); s->hOrdCap = nP * 2; }
  memset(s->hCnt, 0, sizeof(int32_t) * N);
  for (p = 0; p < nP; p++) {
    int gx = jtrunc(s->px[p] / dx); if (gx < 0) gx = 0; else if (gx >= nx) gx = nx - 1;
    int gy = jtrunc(s->py[p] / dx); if (gy < 0) gy = 0; else if (gy >= ny) gy = ny - 1;
    int gz = jtrunc(s->pz[p] / dx); if (gz < 0) gz = 0; else if (gz >= nz) gz = nz - 1;
    s->hCnt[((long)gz * ny + gy) * nx + gx]++;
  }
  int acc = 0;
  for (c = 0; c < N; c++) { s->hStart[c] = acc; acc += s->hCnt[c]; }
  s->hStart[N] = acc;
  memcpy(s->hCur, s->hStart, sizeof(int32_t) * N);
  for (p = 0; p < nP; p++) {
    int gx = jtrunc(s->px[p] / dx); if (gx < 0) gx = 0; else if (gx >= nx) gx = nx - 1;
    int gy = jtrunc(s->py[p] / dx); if (gy < 0) gy = 0; else if (gy >= ny) gy = ny - 1;
    int gz = jtrunc(s->pz[p] / dx); if (gz < 0) gz = 0; else if (gz >= nz) gz = nz - 1;
    c = (int)(((long)gz * ny + gy) * nx + gx);
    s->hOrd[s->hCur[c]++] = p;
  }
  /* shadows + heating (:2773-2918) */
  double cx = s->cx, cy = s->cy, cz = s->cz, coreR2 = s->S.coreR * s->S.coreR;
  long sj = nx + 1, sk = (long)(ny + 1) * sj;
  double Tamb = s->P.Tamb, sunPow = s->P.sunActivity / 3, dissip = 0.045, shadeCool = s->P.shadeCool;
  double half = dx, marchMax = 0.55, absK = 1.1; int marchMaxN = 6;
  const uint8_t* type = s->cellType;
  int sun = s->P.hasSun;
  for (p = 0; p < nP; p++) {
    double lit = sun ? 1 : 0;
    double PX = s->px[p], PY = s->py[p], PZ = s->pz[p];
    double dwx = PX - cx, dwy = PY - cy, dwz = PZ - cz;
    double dwl = sqrt(dwx * dwx + dwy * dwy + dwz * dwz); if (dwl == 0) dwl = 1e-9;
    double stpU = dx / dwl; int above = 0;
    for (int stU = 1; stU <= 4; stU++) {
      double qxU = PX + dwx * stpU * stU, qyU = PY + dwy * stpU * stU, qzU = PZ + dwz * stpU * stU;
      int qiU = jtrunc(qxU / dx), qjU = jtrunc(qyU / dx), qkU = jtrunc(qzU / dx);
      if (qiU < 0 || qjU < 0 || qkU < 0 || qiU >= nx || qjU >= ny || qkU >= nz) break;
      if (type[((long)qkU * ny + qjU) * nx + qiU] != FLUID) break;
      above++;
    }
    s->pDepth[p] = (uint8_t)above;
    if (sun) {
      if (above >= 4) lit = 0;
      else {
        double lx = s->P.sunPos[0] - PX, ly = s->P.sunPos[1] - PY, lz = s->P.sunPos[2] - PZ;
        double ld = sqrt(lx * lx + ly * ly + lz * lz); if (ld == 0) ld = 1e-9;
        double dxn = lx / ld, dyn = ly / ld, dzn = lz / ld;
        double ex = cx - PX, ey = cy - PY, ez = cz - PZ;
        double b = ex * dxn + ey * dyn + ez * dzn;
        if (s->hasTerr) {
          double d2c = ex * ex + ey * ey + ez * ez - b * b;
          if (b > 0 && d2c < s->Rlo2 * 0.96) lit = 0;
          else if (b > 0 || d2c < s->Rhi2 * 1.1) {
            double stp = dx * 1.5, mx = PX, my = PY, mz = PZ;
            double esc2 = (s->Rhi + 0.1) * (s->Rhi + 0.1);
            int tvn = s->tn; double tvd = s->tdv;
            for (int st2 = 0; st2 < 26; st2++) {
              mx += dxn * stp; my += dyn * stp; mz += dzn * stp;
              double rex = mx - cx, rey = my - cy, rez = mz - cz;
              if (rex * rex + rey * rey + rez * rez > esc2) break;
              int ivx = jtrunc(mx / tvd); if (ivx < 0 || ivx >= tvn) break;
              int ivy = jtrunc(my / tvd); if (ivy < 0 || ivy >= tvn) break;
              int ivz = jtrunc(mz / tvd); if (ivz < 0 || ivz >= tvn) break;
              if (s->tsolid[((size_t)ivz * tvn + ivy) * tvn + ivx]) { lit = 0; break; }
            }
          }
        } else if (b > 0) {
          double d2c2 = ex * ex + ey * ey + ez * ez - b * b;
          if (d2c2 < coreR2) lit = 0;
        }
        if (lit) {
          double od = 0, sx = PX, sy = PY, sz = PZ;
          for (int st = 0; st < marchMaxN && st * half < marchMax; st++) {
            sx += dxn * half; sy += dyn * half; sz += dzn * half;
            int i0 = jtrunc(sx / dx), j0 = jtrunc(sy / dx), k0 = jtrunc(sz / dx);
            if (i0 < 0 || j0 < 0 || k0 < 0 || i0 >= nx || j0 >= ny || k0 >= nz) break;
            double vv = s->dens[k0 * sk + j0 * sj + i0];
            od += vv * half * absK;
            if (od > 3.5) break;
          }
          if (od < 3.5) lit = exp(-od); else lit = 0;
        }
      }
    }
    s->pLight[p] = (st_t)lit;
    double T, pT = s->pT[p]; int f = s->pflag[p];
    if (f == 2) {
      double airAmb = lit > 0.05 ? Tamb + 0.18 : 0.06;
      double airK = sun ? 0.16 + (1 - lit) * 0.20 : 1.2;
      T = pT + (airAmb - pT) * airK * dt;
      if (lit > 0) T += sunPow * 0.6 * lit * dt;
    } else if (f == 3) {
      double cldAmb = lit > 0.05 ? Tamb + 0.18 : 0.06;
      double cldK = sun ? 0.10 + (1 - lit) * 0.12 : 0.9;
      T = pT + (cldAmb - pT) * cldK * dt;
      if (lit > 0) T += sunPow * 0.35 * lit * dt;
    } else if (f == 4) {
      double rainAmb = lit > 0.05 ? Tamb + 0.18 : 0.06;
      double rainK = sun ? 0.14 + (1 - lit) * 0.16 : 1.0;
      T = pT + (rainAmb - pT) * rainK * dt;
      if (lit > 0) T += sunPow * 0.45 * lit * dt;
    } else {
      double watAmb = lit > 0.05 ? Tamb : 0;
      T = pT + (watAmb - pT) * (dissip + (1 - lit) * shadeCool) * dt;
      if (lit > 0) T += sunPow * lit * dt;
    }
    if (T > 1.15) T = 1.15; else if (T < 0) T = 0;
    s->pT[p] = (st_t)T;
  }
  if (s->P.heatK > 0) {
    /* means (:2921-2934), flux (:2938-2964), apply (:2966-2979) */
    for (c = 0; c < N; c++) {
      double sumT = 0;
      for (int e = s->hStart[c]; e < s->hStart[c + 1]; e++) sumT += s->pT[s->hOrd[e]];
      s->heatMean[c] = s->hCnt[c] ? sumT / s->hCnt[c] : 0;
    }
    double alpha = jmin(s->P.heatK * s->heatDt * 0.15, 0.14);
    memset(s->heatDelta, 0, sizeof(double) * N);
    long nxyH = (long)nx * ny; int i, j, k;
    for (k = 0; k < nz; k++) for (j = 0; j < ny; j++) for (i = 0; i < nx; i++) {
      c = (int)(((long)k * ny + j) * nx + i);
      if (!s->hCnt[c]) continue;
      for (int axis = 0; axis < 3; axis++) {
        if ((axis == 0 && i == nx - 1) || (axis == 1 && j == ny - 1) || (axis == 2 && k == nz - 1)) continue;
        long nbr = c + (axis == 0 ? 1 : axis == 1 ? nx : nxyH);
        if (!s->hCnt[nbr]) continue;
        double energy = alpha * (double)(s->hCnt[c] < s->hCnt[nbr] ? s->hCnt[c] : s->hCnt[nbr]) *
                        (s->heatMean[nbr] - s->heatMean[c]);
        s->heatDelta[c] += energy; s->heatDelta[nbr] -= energy;
      }
    }
    double alphaA = s->heatAlpha;
    for (c = 0; c < N; c++) {
      if (!s->hCnt[c]) continue;
      double deltaT = s->heatDelta[c] / s->hCnt[c];
      for (int e = s->hStart[c]; e < s->hStart[c + 1]; e++) {
        int q = s->hOrd[e];
        s->pT[q] = (st_t)(s->pT[q] + alphaA * (s->heatMean[c] - s->pT[q]) + deltaT);
      }
    }
  }
  /* convection (:2982-2994) */
  double beta = 3.0;
  for (p = 0; p < nP; p++) {
    if (s->pflag[p] != 0) continue;
    double rx = s->px[p] - cx, ry = s->py[p] - cy, rz = s->pz[p] - cz;
    double rl = sqrt(rx * rx + ry * ry + rz * rz); if (rl == 0) rl = 1e-9;
    double ab = beta * ((double)s->pT[p] - Tamb) * dt / rl;
    s->pvx[p] += rx * ab; s->pvy[p] += ry * ab; s->pvz[p] += rz * ab;
  }
}

/* ------------------------------------------------------------ evaporation
 * _updateEvaporation/_evapChunk/_evGauss, js/solver.js:3008-3125 */
static double ev_gauss(or_solver* s) {
  double u1;
  do { s->S.evS = lcg(s->S.evS); u1 = s->S.evS / 4294967296.0; } while (u1 < 1e-9);
  s->S.evS = lcg(s->S.evS);
  return sqrt(-2 * log(u1)) * cos(6.283185306 * (s->S.evS / 4294967296.0));
}
void or_update_evaporation(or_solver* s, double dt) {
  if (s->P.sunActivity <= 0 || s->P.evapIntensity <= 0) return;
  double rate = s->P.sunActivity * s->P.evapIntensity;
  int evapN = 0;
  if (rate > 0) {
    double freezeT = jmax(s->P.meltT, s->P.snowT * 1.05);
    int nx = s->nx, ny = s->ny, nz = s->nz, nP = s->S.nP; double dx = s->dx;
    double cx = s->cx, cy = s->cy, cz = s->cz, C = EVAP_STEEPNESS, T_CAP = 1.15;
    const uint8_t* type = s->cellType;
    for (int p = 0; p < nP; p++) {
      if (s->pflag[p] != 0) continue;
      double T = s->pT[p];
      if (T <= freezeT) continue;
      double PX = s->px[p], PY = s->py[p], PZ = s->pz[p];
      int i = jtrunc(PX / dx), j = jtrunc(PY / dx), k = jtrunc(PZ / dx);
      if (i < 1) i = 1; else if (i > nx - 2) i = nx - 2;
      if (j < 1) j = 1; else if (j > ny - 2) j = ny - 2;
      if (k < 1) k = 1; else if (k > nz - 2) k = nz - 2;
      long c = ((long)k * ny + j) * nx + i;
      if (type[c] != FLUID) continue;
      double ex = PX - cx, ey = PY - cy, ez = PZ - cz;
      double el = sqrt(ex * ex + ey * ey + ez * ez); if (el == 0) el = 1e-9;
      int ui = jtrunc((PX + ex / el * dx) / dx), uj = jtrunc((PY + ey / el * dx) / dx), uk = jtrunc((PZ + ez / el * dx) / dx);
      if (ui < 0 || uj < 0 || uk < 0 || ui >= nx || uj >= ny || uk >= nz) continue;
      if (type[((long)uk * ny + uj) * nx + ui] == FLUID) continue;
      double tau = (T - freezeT) / (T_CAP - freezeT);
      if (tau < 0) tau = 0; else if (tau > 1) tau = 1;
      double prob = rate * dt * exp(C * (T - freezeT));
      if (prob > 1) prob = 1;
      s->S.evS = lcg(s->S.evS);
      double rnd = s->S.evS / 4294967296.0;
      if (rnd > prob) continue;
      s->pflag[p] = 2; s->pAir[p] = 0;
      double sig = 0.30 + 0.32 * sqrt(tau);
      double kx = sig * ev_gauss(s); double ky = sig * ev_gauss(s); double kz = sig * ev_gauss(s);
      double ex2 = PX - cx, ey2 = PY - cy, ez2 = PZ - cz;
      double el2 = ex2 * ex2 + ey2 * ey2 + ez2 * ez2;
      double elL = sqrt(el2); if (elL == 0) elL = 1e-9;
      double kUp = (kx * ex2 + ky * ey2 + kz * ez2) / el2;
      if (kUp < 0) { kx -= 2 * kUp * ex2 / elL; ky -= 2 * kUp * ey2 / elL; kz -= 2 * kUp * ez2 / elL; }
      double guS = s->u[((long)k * ny + j) * (nx + 1) + i];
      double gvS = s->v[((long)k * (ny + 1) + j) * nx + i];
      double gwS = s->w[((long)k * ny + j) * nx + i];
      double nl2 = 1 / el2, vN = ((double)s->pvx[p] * ex2 + (double)s->pvy[p] * ey2 + (double)s->pvz[p] * ez2) * nl2;
      double vNx = vN * ex2, vNy = vN * ey2, vNz = vN * ez2;
      double gN = (guS * ex2 + gvS * ey2 + gwS * ez2) * nl2;
      double vtx = guS - gN * ex2, vty = gvS - gN * ey2, vtz = gwS - gN * ez2;
      s->pvx[p] = (st_t)(vNx + vtx + kx); s->pvy[p] = (st_t)(vNy + vty + ky); s->pvz[p] = (st_t)(vNz + vtz + kz);
      evapN++;
    }
  }
  s->S.evapCount = evapN;
}

/* ------------------------------------------------------------ phases
 * _spinHash + _updatePhaseChanges, js/solver.js:3145-3281 */
static uint32_t js_mul_u32(double a, double b) {       /* (a*b) as a JS double, then ToUint32 */
  double d = a * b;
  double m = fmod(d, 4294967296.0); if (m < 0) m += 4294967296.0;
  return (uint32_t)m;
}
static uint32_t spin_hash(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t s = a ^ js_mul_u32(b, 0x9e3779b9) ^ js_mul_u32(c, 0x85ebca6b) ^ js_mul_u32(0x51ab3c77, 0xc2b2ae35);
  s = lcg(s);
  s ^= s >> 13; s = js_mul_u32(s, 0x5bd1e995); s ^= s >> 15;
  return s;
}
void or_update_phase(or_solver* s, double dt) {
  int nP = s->S.nP, nx = s->nx, ny = s->ny, nz = s->nz, p, i, j, k; double dx = s->dx;
  int32_t* cnt = s->steamCnt;
  memset(cnt, 0, sizeof(int32_t) * s->nCells);
  for (p = 0; p < nP; p++) {
    if (s->pflag[p] != 2) continue;
    i = jtrunc(s->px[p] / dx); j = jtrunc(s->py[p] / dx); k = jtrunc(s->pz[p] / dx);
    if (i < 0) i = 0; else if (i >= nx) i = nx - 1;
    if (j < 0) j = 0; else if (j >= ny) j = ny - 1;
    if (k < 0) k = 0; else if (k >= nz) k = nz - 1;
    cnt[((long)k * ny + j) * nx + i]++;
  }
  double cloudT = s->P.cloudT, cloudP = s->P.cloudP;
  double rainT = jmin(s->P.rainT, cloudT - 0.02); if (rainT < 0) rainT = 0;
  double snowT = jmin(s->P.snowT, rainT - 0.02); if (snowT < 0) snowT = 0;
  double meltT = s->P.meltT > snowT * 1.05 ? s->P.meltT : snowT * 1.05;
  const uint8_t* type = s->cellType;
  double cloudBase = s->S.oceanR + 0.3 * s->P.atmosphereH;
  double cx = s->cx, cy = s->cy, cz = s->cz;
  long nxy = (long)nx * ny;
  for (p = 0; p < nP; p++) {
    int f = s->pflag[p];
    if (f == 0) {
      if (s->pT[p] <= snowT && s->pT[p] > 1e-3) {
        i = jtrunc(s->px[p] / dx); j = jtrunc(s->py[p] / dx); k = jtrunc(s->pz[p] / dx);
        if (i < 0) i = 0; else if (i >= nx) i = nx - 1;
        if (j < 0) j = 0; else if (j >= ny) j = ny - 1;
        if (k < 0) k = 0; else if (k >= nz) k = nz - 1;
        long cB = ((long)k * ny + j) * nx + i;
        int atSurf = (k > 0 && type[cB - nxy] != FLUID) || (k < nz - 1 && type[cB + nxy] != FLUID) ||
                     (j > 0 && type[cB - nx] != FLUID) || (j < ny - 1 && type[cB + nx] != FLUID) ||
                     (i > 0 && type[cB - 1] != FLUID) || (i < nx - 1 && type[cB + 1] != FLUID);
        if (atSurf) { s->pflag[p] = 5; s->pvx[p] = s->pvy[p] = s->pvz[p] = 0; s->pAir[p] = 1; }
      }
      continue;
    }
    if (f == 5) {
      if (s->pT[p] >= meltT) {
        i = jtrunc(s->px[p] / dx); j = jtrunc(s->py[p] / dx); k = jtrunc(s->pz[p] / dx);
        if (i < 0) i = 0; else if (i >= nx) i = nx - 1;
        if (j < 0) j = 0; else if (j >= ny) j = ny - 1;
        if (k < 0) k = 0; else if (k >= nz) k = nz - 1;
        s->pflag[p] = type[((long)k * ny + j) * nx + i] == FLUID ? 0 : 4;
        s->pAir[p] = 0;
        s->pWx[p] = s->pWy[p] = s->pWz[p] = 0;
      }
      continue;
    }
    double T = s->pT[p];
    if (T <= 1e-3) continue;
    if (f == 2) {
      if (T <= rainT && s->pAir[p] >= s->P.rainLiftAge) {
        s->pflag[p] = 4; s->pAir[p] = 0;
        s->pvx[p] = s->pvy[p] = s->pvz[p] = 0;
        s->pWx[p] = s->pWy[p] = s->pWz[p] = 0;
        continue;
      }
      if (T > cloudT) continue;
      double rx = (double)s->px[p] - cx, ry = (double)s->py[p] - cy, rz = (double)s->pz[p] - cz;
      if (sqrt(rx * rx + ry * ry + rz * rz) < cloudBase) continue;
      i = jtrunc(s->px[p] / dx); j = jtrunc(s->py[p] / dx); k = jtrunc(s->pz[p] / dx);
      int i0 = i > 0 ? i - 1 : 0, i1 = i < nx - 1 ? i + 1 : nx - 1;
      int j0 = j > 0 ? j - 1 : 0, j1 = j < ny - 1 ? j + 1 : ny - 1;
      int k0 = k > 0 ? k - 1 : 0, k1 = k < nz - 1 ? k + 1 : nz - 1;
      double sum = 0;
      for (int kk = k0; kk <= k1; kk++) for (int jj = j0; jj <= j1; jj++) {
        long row = ((long)kk * ny + jj) * nx;
        for (int ii = i0; ii <= i1; ii++) sum += cnt[row + ii];
      }
      if (sum / 27 >= cloudP) { s->pflag[p] = 3; s->pAir[p] = 0; }
      continue;
    }
    if (f == 3) { if (T >= cloudT + 0.05) s->pflag[p] = 2; continue; }
    if (T <= snowT) {
      s->pflag[p] = 5; s->pvx[p] = s->pvy[p] = s->pvz[p] = 0; s->pAir[p] = 0;
      s->pWx[p] = s->pWy[p] = s->pWz[p] = 0;
    }
  }
  if (s->P.spinOn && dt > 0) {
    uint32_t tick = (uint32_t)jtrunc(s->S.simTime * 60), sd = 0x51ab3c77u;
    double damp = jmax(0, 1 - 0.12 * dt);
    for (p = 0; p < nP; p++) {
      int f = s->pflag[p];
      if (f != 2 && f != 3) continue;
      if (f == 2 && s->pAir[p] <= 1e-6 && s->pWx[p] == 0 && s->pWy[p] == 0 && s->pWz[p] == 0) {
        double h1 = spin_hash(sd, (uint32_t)p, tick) / 4294967296.0;
        double h2 = spin_hash(sd + 1, (uint32_t)p, tick) / 4294967296.0;
        double h3 = spin_hash(sd + 2, (uint32_t)p, tick) / 4294967296.0;
        double zz = 2 * h2 - 1, rr = sqrt(jmax(0, 1 - zz * zz)), th = 6.283185306 * h1;
        double Tp = s->pT[p]; if (!(Tp > 0.05)) Tp = 0.05; else if (Tp > 1.15) Tp = 1.15;
        double wSpd = 3.0 * sqrt(Tp) * (0.5 + h3);
        s->pWx[p] = (st_t)(rr * cos(th) * wSpd); s->pWy[p] = (st_t)(zz * wSpd); s->pWz[p] = (st_t)(rr * sin(th) * wSpd);
      }
      double wm = sqrt((double)s->pWx[p] * s->pWx[p] + (double)s->pWy[p] * s->pWy[p] + (double)s->pWz[p] * s->pWz[p]);
      if (wm > 1e-6) s->pPh[p] += wm * dt;
      s->pWx[p] *= damp; s->pWy[p] *= damp; s->pWz[p] *= damp;
    }
  }
}

/* ------------------------------------------------------------ contacts
 * sort order of js/solver.js:3303/3370: px ascending, then index */
static const st_t* g_sort_px;
static int cmp_px_idx(const void* A, const void* B) {
  int a = *(const int32_t*)A, b = *(const int32_t*)B;
  double d = (double)g_sort_px[a] - g_sort_px[b];
  if (d < 0) return -1;
  if (d > 0) return 1;
  return a < b ? -1 : (a > b ? 1 : 0);
}
static void ensure_idx(or_solver* s, int n) {
  if (s->idxCap >= n) return;
  free(s->vIdx); free(s->iceIdx);
  s->vIdx = xcalloc(n, sizeof(int32_t)); s->iceIdx = xcalloc(n, sizeof(int32_t)); s->idxCap = n;
}

/* _iceContacts, js/solver.js:3290-3324 */
void or_ice_contacts(or_solver* s) {
  int nP = s->S.nP, nI = 0, p;
  ensure_idx(s, nP > 0 ? nP : 1);
  for (p = 0; p < nP; p++) if (s->pflag[p] == 5) s->iceIdx[nI++] = p;
  if (nI < 2) return;
  double rad = s->S.spacing * 0.7, rad2 = rad * rad;
  g_sort_px = s->px; qsort(s->iceIdx, nI, sizeof(int32_t), cmp_px_idx);
  st_t *px = s->px, *py = s->py, *pz = s->pz, *pvx = s->pvx, *pvy = s->pvy, *pvz = s->pvz, *pAir = s->pAir;
  for (int a = 0; a < nI; a++) {
    int i = s->iceIdx[a];
    int stuckI = pAir[i] == 1;
    for (int b = a + 1; b < nI; b++) {
      int j = s->iceIdx[b];
      if ((double)px[j] - px[i] >= rad) break;
      double ddx = (double)px[j] - px[i], ddy = (double)py[j] - py[i], ddz = (double)pz[j] - pz[i];
      if (ddx * ddx + ddy * ddy + ddz * ddz >= rad2) continue;
      int stuckJ = pAir[j] == 1;
      if (stuckI && stuckJ) continue;
      if (stuckJ) { pAir[i] = 1; pvx[i] = pvy[i] = pvz[i] = 0; stuckI = 1; }
      else if (stuckI) { pAir[j] = 1; pvx[j] = pvy[j] = pvz[j] = 0; }
      else {
        double mx = ((double)pvx[i] + pvx[j]) * 0.5, my = ((double)pvy[i] + pvy[j]) * 0.5, mz = ((double)pvz[i] + pvz[j]) * 0.5;
        pvx[i] = pvx[j] = (st_t)mx; pvy[i] = pvy[j] = (st_t)my; pvz[i] = pvz[j] = (st_t)mz;
      }
    }
  }
}

/* _vaporCollisions, js/solver.js:3345-3479 */
void or_vapor_collisions(or_solver* s) {
  int nP = s->S.nP, nV = 0, night = 0, nSteam = 0, p;
  ensure_idx(s, nP > 0 ? nP : 1);
  int sun = s->P.hasSun;
  double sx = sun ? s->P.sunPos[0] - s->cx : 0, sy = sun ? s->P.sunPos[1] - s->cy : 0, sz = sun ? s->P.sunPos[2] - s->cz : 0;
  for (p = 0; p < nP; p++) {
    int fp = s->pflag[p];
    if (fp != 2 && fp != 3) continue;
    s->vIdx[nV++] = p;
    if (fp == 2) {
      nSteam++;
      if (!sun || ((double)s->px[p] - s->cx) * sx + ((double)s->py[p] - s->cy) * sy + ((double)s->pz[p] - s->cz) * sz < 0) night++;
    }
  }
  s->S.vaporCount = nSteam; s->S.nightVaporCount = night;
  if (nV < 2) return;
  st_t *px = s->px, *py = s->py, *pz = s->pz, *pvx = s->pvx, *pvy = s->pvy, *pvz = s->pvz;
  st_t *pWx = s->pWx, *pWy = s->pWy, *pWz = s->pWz;
  int spinOn = s->P.spinOn;
  double rad = s->S.spacing * 0.6, rad2 = rad * rad;
  int32_t* vIdx = s->vIdx;
  g_sort_px = px; qsort(vIdx, nV, sizeof(int32_t), cmp_px_idx);
  for (int a = 0; a < nV; a++) {
    int i = vIdx[a];
    for (int b = a + 1; b < nV; b++) {
      int j = vIdx[b];
      if ((double)px[j] - px[i] >= rad) break;
      double ddx = (double)px[j] - px[i], ddy = (double)py[j] - py[i], ddz = (double)pz[j] - pz[i];
      double d2 = ddx * ddx + ddy * ddy + ddz * ddz;
      if (d2 >= rad2) continue;
      double d = sqrt(d2); if (d == 0) d = 1e-9;
      double nX = ddx / d, nY = ddy / d, nZ = ddz / d;
      double vRel = ((double)pvx[i] - pvx[j]) * nX + ((double)pvy[i] - pvy[j]) * nY + ((double)pvz[i] - pvz[j]) * nZ;
      if (vRel > 0) {
        pvx[i] -= vRel * nX; pvy[i] -= vRel * nY; pvz[i] -= vRel * nZ;
        pvx[j] += vRel * nX; pvy[j] += vRel * nY; pvz[j] += vRel * nZ;
      }
      double half = (rad - d) * 0.5;
      px[i] -= nX * half; py[i] -= nY * half; pz[i] -= nZ * half;
      px[j] += nX * half; py[j] += nY * half; pz[j] += nZ * half;
      double kick = (rad - d) * 2;
      pvx[i] -= nX * kick; pvy[i] -= nY * kick; pvz[i] -= nZ * kick;
      pvx[j] += nX * kick; pvy[j] += nY * kick; pvz[j] += nZ * kick;
      if (!spinOn) continue;
      double R = rad * 0.5;
      double wSx = (double)pWx[i] + pWx[j], wSy = (double)pWy[i] + pWy[j], wSz = (double)pWz[i] + pWz[j];
      double usx = ((double)pvx[i] - pvx[j]) + R * (wSy * nZ - wSz * nY);
      double usy = ((double)pvy[i] - pvy[j]) + R * (wSz * nX - wSx * nZ);
      double usz = ((double)pvz[i] - pvz[j]) + R * (wSx * nY - wSy * nX);
      double uN = usx * nX + usy * nY + usz * nZ;
      double utx = usx - uN * nX, uty = usy - uN * nY, utz = usz - uN * nZ;
      double utM = sqrt(utx * utx + uty * uty + utz * utz);
      if (utM < 1e-9) continue;
      double jt = utM / 7;
      if (vRel > 0) { double mu = 0.25 * vRel; if (jt > mu) jt = mu; }
      double jx = -utx / utM * jt, jy = -uty / utM * jt, jz = -utz / utM * jt;
      pvx[i] += jx; pvy[i] += jy; pvz[i] += jz;
      pvx[j] -= jx; pvy[j] -= jy; pvz[j] -= jz;
      double invI = 1 / (0.4 * R * R);
      double dwx = R * (nY * jz - nZ * jy) * invI, dwy = R * (nZ * jx - nX * jz) * invI, dwz = R * (nX * jy - nY * jx) * invI;
      pWx[i] += dwx; pWy[i] += dwy; pWz[i] += dwz;
      pWx[j] += dwx; pWy[j] += dwy; pWz[j] += dwz;
    }
  }
  double dxc = s->dx;
  double band = s->S.oceanR - dxc * 2, bandLo2 = band * band;
  double radW = rad, radW2 = rad2;
  for (p = 0; p < nP; p++) {
    int fw = s->pflag[p];
    if (fw != 0 && fw != 1 && fw != 4) continue;
    double wx = px[p], wy = py[p], wz = pz[p];
    if (fw == 0) {
      double dwx2 = wx - s->cx, dwy2 = wy - s->cy, dwz2 = wz - s->cz;
      if (dwx2 * dwx2 + dwy2 * dwy2 + dwz2 * dwz2 < bandLo2) continue;
    }
    int lo = 0, hi = nV;
    while (lo < hi) { int mid = (lo + hi) >> 1; if ((double)px[vIdx[mid]] < wx - radW) lo = mid + 1; else hi = mid; }
    for (int b2 = lo; b2 < nV; b2++) {
      int j2 = vIdx[b2];
      double ddx2 = (double)px[j2] - wx;
      if (ddx2 >= radW) break;
      double ddy2 = (double)py[j2] - wy, ddz2 = (double)pz[j2] - wz;
      double dd2 = ddx2 * ddx2 + ddy2 * ddy2 + ddz2 * ddz2;
      if (dd2 >= radW2 || dd2 < 1e-12) continue;
      double dd = sqrt(dd2);
      double nX2 = ddx2 / dd, nY2 = ddy2 / dd, nZ2 = ddz2 / dd;
      double vR2 = ((double)pvx[j2] - pvx[p]) * nX2 + ((double)pvy[j2] - pvy[p]) * nY2 + ((double)pvz[j2] - pvz[p]) * nZ2;
      if (vR2 < 0) { double vB = vR2 * (1 + 0.4); pvx[j2] -= vB * nX2; pvy[j2] -= vB * nY2; pvz[j2] -= vB * nZ2; }
      double ov2 = radW - dd;
      px[j2] += nX2 * ov2; py[j2] += nY2 * ov2; pz[j2] += nZ2 * ov2;
      double kk2 = ov2 * 2;
      pvx[j2] += nX2 * kk2; pvy[j2] += nY2 * kk2; pvz[j2] += nZ2 * kk2;
    }
  }
}

/* _pushSurfaceChunk, js/solver.js:3496-3587 */
void or_push_surface(or_solver* s) {
  if (!s->hasTerr) return;
  int nP = s->S.nP; double cx = s->cx, cy = s->cy, cz = s->cz, dx = s->dx;
  st_t *px = s->px, *py = s->py, *pz = s->pz, *pvx = s->pvx, *pvy = s->pvy, *pvz = s->pvz;
  for (int p = 0; p < nP; p++) {
    double x = px[p], y = py[p], z = pz[p];
    double ex = x - cx, ey = y - cy, ez = z - cz;
    double er = sqrt(ex * ex + ey * ey + ez * ez); if (er == 0) er = 1e-9;
    int fixed = 0, rockFixed = 0;
    double outer = s->domainR - dx * 0.02;
    double skyHi = s->S.oceanR + s->P.atmosphereH - 1e-3 * dx;
    if (er > skyHi) {
      x = cx + ex / er * skyHi; y = cy + ey / er * skyHi; z = cz + ez / er * skyHi;
      double outward = ((double)pvx[p] * ex + (double)pvy[p] * ey + (double)pvz[p] * ez) / er;
      if (outward > 0) { pvx[p] -= ex / er * outward; pvy[p] -= ey / er * outward; pvz[p] -= ez / er * outward; }
      px[p] = (st_t)x; py[p] = (st_t)y; pz[p] = (st_t)z;
      ex = x - cx; ey = y - cy; ez = z - cz; er = skyHi;
      fixed = 1;
    }
    if (er <= s->domainR && ROCK(s, x, y, z)) {
      rockFixed = 1;
      int tries = 0;
      while (ROCK(s, x, y, z) && tries < s->nx * 2) {
        x += ex / er * dx * 0.5; y += ey / er * dx * 0.5; z += ez / er * dx * 0.5;
        tries++;
      }
      double exR = x - cx, eyR = y - cy, ezR = z - cz;
      double erR = sqrt(exR * exR + eyR * eyR + ezR * ezR); if (erR == 0) erR = 1e-9;
      double wantR = TRAD(s, x, y, z) + dx * 0.06;
      if (erR > wantR) { x = cx + exR / erR * wantR; y = cy + eyR / erR * wantR; z = cz + ezR / erR * wantR; }
      int kR = 0;
      while (ROCK(s, x, y, z) && kR < 4) {
        x += exR / erR * dx * 0.5; y += eyR / erR * dx * 0.5; z += ezR / erR * dx * 0.5;
        kR++;
      }
      fixed = 1;
    } else if (s->pflag[p] == 0 && er <= s->domainR) {
      double Rt = TRAD(s, x, y, z);
      if (er < Rt - dx * 0.5) {
        rockFixed = 1;
        int t2 = 0;
        x = cx + ex / er * (Rt + dx * 0.05);
        y = cy + ey / er * (Rt + dx * 0.05);
        z = cz + ez / er * (Rt + dx * 0.05);
        while (ROCK(s, x, y, z) && t2 < 8) {
          x += ex / er * dx * 0.5; y += ey / er * dx * 0.5; z += ez / er * dx * 0.5;
          t2++;
        }
        fixed = 1;
      }
    }
    double finalR = sqrt((x - cx) * (x - cx) + (y - cy) * (y - cy) + (z - cz) * (z - cz));
    double capR = s->pflag[p] == 0 ? outer : skyHi;
    if (finalR > capR) {
      x = cx + (x - cx) * capR / finalR; y = cy + (y - cy) * capR / finalR; z = cz + (z - cz) * capR / finalR;
      fixed = 1;
    }
    if (fixed) {
      px[p] = (st_t)x; py[p] = (st_t)y; pz[p] = (st_t)z;
      double vr = ((double)pvx[p] * ex + (double)pvy[p] * ey + (double)pvz[p] * ez) / er;
      if (rockFixed && vr < 0) { pvx[p] -= ex / er * vr; pvy[p] -= ey / er * vr; pvz[p] -= ez / er * vr; }
    }
  }
}

/* ------------------------------------------------------------ surface
 * splatDensity/_splatInto, js/solver.js:3785-3820 */
void or_splat_density(or_solver* s) {
  int nx = s->nx, ny = s->ny, nz = s->nz, nP = s->S.nP; double dx = s->dx;
  long nd = (long)(nx + 1) * (ny + 1) * (nz + 1);
  memset(s->dens, 0, sizeof(st_t) * nd);
  double r = 1.6 * s->S.spacing, r2 = r * r;
  long sj = nx + 1, sk = (long)(ny + 1) * sj;
  for (int p = 0; p < nP; p++) {
    if (s->pflag[p] != 0) continue;
    double gx = s->px[p] / dx, gy = s->py[p] / dx, gz = s->pz[p] / dx;
    double fi = floor(gx), fj = floor(gy), fk = floor(gz);
    int i0 = fi < 0 ? 0 : (fi > nx - 1 ? nx - 1 : (int)fi);
    int j0 = fj < 0 ? 0 : (fj > ny - 1 ? ny - 1 : (int)fj);
    int k0 = fk < 0 ? 0 : (fk > nz - 1 ? nz - 1 : (int)fk);
    double fx = s->px[p] - i0 * dx, fy = s->py[p] - j0 * dx, fz = s->pz[p] - k0 * dx;
    for (int kk = 0; kk < 2; kk++) {
      double czz = kk == 0 ? fz : fz - dx;
      for (int jj = 0; jj < 2; jj++) {
        double cyy = jj == 0 ? fy : fy - dx;
        for (int ii = 0; ii < 2; ii++) {
          double cxx = ii == 0 ? fx : fx - dx;
          double d2 = cxx * cxx + cyy * cyy + czz * czz;
          if (d2 >= r2) continue;
          double ww = 1 - d2 / r2; ww = ww * ww;
          s->dens[(k0 + kk) * sk + (j0 + jj) * sj + (i0 + ii)] += ww;
        }
      }
    }
  }
}

/* MarchingTetrahedra.build, js/surface.js:17-177: triangle count, signed-
 * volume integral and, when pos/nrm are given, the emitted vertices (float
 * positions and gradient normals, 3 per vertex, in cell/tet/case order, at
 * most maxVerts) */
static const int MT_CORNERS[8][3] = { {0,0,0},{1,0,0},{1,1,0},{0,1,0},{0,0,1},{1,0,1},{1,1,1},{0,1,1} };
static const int MT_TETS[6][4] = { {0,5,1,6},{0,1,2,6},{0,2,3,6},{0,3,7,6},{0,7,4,6},{0,4,5,6} };
static const int MT_EDGES[6][2] = { {0,1},{1,2},{2,0},{0,3},{1,3},{2,3} };
static const int MT_NTRI[16] = { 0,1,1,2,1,2,2,1,1,2,2,1,2,1,1,0 };
static const int MT_CASES[16][2][3] = {
  {{0,0,0},{0,0,0}}, {{0,2,3},{0,0,0}}, {{0,1,4},{0,0,0}}, {{2,3,4},{2,4,1}},
  {{2,1,5},{0,0,0}}, {{0,3,5},{0,5,1}}, {{0,4,5},{0,5,2}}, {{3,5,4},{0,0,0}},
  {{3,4,5},{0,0,0}}, {{0,2,5},{0,5,4}}, {{0,1,5},{0,5,3}}, {{2,1,5},{0,0,0}},
  {{2,1,4},{2,4,3}}, {{0,1,4},{0,0,0}}, {{0,2,3},{0,0,0}}, {{0,0,0},{0,0,0}} };
static double mt_volume_impl(const st_t* dens, int nx, int ny, int nz, double dx, double iso, int64_t* triCount,
                             float* pos, float* nrm, int64_t maxVerts) {
  long sj = nx + 1, sk = (long)(ny + 1) * sj;
  double volume = 0; int64_t vcount = 0;
  double cv[8], gx[8], gy[8], gz[8], tv[4];
  for (int k = 0; k < nz; k++) for (int j = 0; j < ny; j++) for (int i = 0; i < nx; i++) {
    double minv = INFINITY, maxv = -INFINITY;
    for (int c = 0; c < 8; c++) {
      double val = dens[(k + MT_CORNERS[c][2]) * sk + (j + MT_CORNERS[c][1]) * sj + (i + MT_CORNERS[c][0])];
      cv[c] = val; if (val < minv) minv = val; if (val > maxv) maxv = val;
    }
    if (maxv < iso || minv > iso) continue;
    for (int c = 0; c < 8; c++) {
      int ci = i + MT_CORNERS[c][0], cj = j + MT_CORNERS[c][1], ck = k + MT_CORNERS[c][2];
      int ip = ci + 1 < nx ? ci + 1 : nx, im = ci - 1 > 0 ? ci - 1 : 0;
      int jp = cj + 1 < ny ? cj + 1 : ny, jm = cj - 1 > 0 ? cj - 1 : 0;
      int kp = ck + 1 < nz ? ck + 1 : nz, km = ck - 1 > 0 ? ck - 1 : 0;
      gx[c] = ((double)dens[ck * sk + cj * sj + ip] - dens[ck * sk + cj * sj + im]) / (2 * dx);
      gy[c] = ((double)dens[ck * sk + jp * sj + ci] - dens[ck * sk + jm * sj + ci]) / (2 * dx);
      gz[c] = ((double)dens[kp * sk + cj * sj + ci] - dens[km * sk + cj * sj + ci]) / (2 * dx);
    }
    for (int t = 0; t < 6; t++) {
      const int* tet = MT_TETS[t]; int code = 0;
      for (int c = 0; c < 4; c++) { tv[c] = cv[tet[c]]; if (tv[c] > iso) code |= (1 << c); }
      int ntri = MT_NTRI[code];
      for (int e = 0; e < ntri; e++) {
        double P3[3][3], N3[3][3];
        for (int vi = 0; vi < 3; vi++) {
          int ed = MT_CASES[code][e][vi];
          int a = tet[MT_EDGES[ed][0]], b = tet[MT_EDGES[ed][1]];
          double va = cv[a], vb = cv[b], den = vb - va;
          double tt = den != 0 ? (iso - va) / den : 0.5;
          if (tt < 0) tt = 0; else if (tt > 1) tt = 1;
          const int *pa = MT_CORNERS[a], *pb = MT_CORNERS[b];
          double wxx = (i + pa[0]) + (pb[0] - pa[0]) * tt;
          double wyy = (j + pa[1]) + (pb[1] - pa[1]) * tt;
          double wzz = (k + pa[2]) + (pb[2] - pa[2]) * tt;
          P3[vi][0] = wxx * dx; P3[vi][1] = wyy * dx; P3[vi][2] = wzz * dx;   /* px3/py3/pz3: plain JS arrays */
          double nxx = -(gx[a] + (gx[b] - gx[a]) * tt);
          double nyy = -(gy[a] + (gy[b] - gy[a]) * tt);
          double nzz = -(gz[a] + (gz[b] - gz[a]) * tt);
          double nl = sqrt(nxx * nxx + nyy * nyy + nzz * nzz); if (nl == 0) nl = 1;
          N3[vi][0] = nxx / nl; N3[vi][1] = nyy / nl; N3[vi][2] = nzz / nl;
        }
        double ux = P3[1][0] - P3[0][0], uy = P3[1][1] - P3[0][1], uz = P3[1][2] - P3[0][2];
        double vx2 = P3[2][0] - P3[0][0], vy2 = P3[2][1] - P3[0][1], vz2 = P3[2][2] - P3[0][2];
        double fnx = uy * vz2 - uz * vy2, fny = uz * vx2 - ux * vz2, fnz = ux * vy2 - uy * vx2;
        double cgx = N3[0][0] + N3[1][0] + N3[2][0];
        double cgy = N3[0][1] + N3[1][1] + N3[2][1];
        double cgz = N3[0][2] + N3[1][2] + N3[2][2];
        if (fnx * cgx + fny * cgy + fnz * cgz < 0) {
          for (int d = 0; d < 3; d++) {
            double tmp = P3[2][d]; P3[2][d] = P3[1][d]; P3[1][d] = tmp;
            tmp = N3[2][d]; N3[2][d] = N3[1][d]; N3[1][d] = tmp;
          }
        }
        volume += (P3[0][0] * (P3[1][1] * P3[2][2] - P3[2][1] * P3[1][2]) -
                   P3[0][1] * (P3[1][0] * P3[2][2] - P3[2][0] * P3[1][2]) +
                   P3[0][2] * (P3[1][0] * P3[2][1] - P3[2][0] * P3[1][1])) / 6;
        if (pos && nrm && vcount + 3 <= maxVerts)
          for (int vi = 0; vi < 3; vi++)
            for (int d = 0; d < 3; d++) { pos[(vcount + vi) * 3 + d] = (float)P3[vi][d]; nrm[(vcount + vi) * 3 + d] = (float)N3[vi][d]; }
        vcount += 3;
      }
    }
  }
  if (triCount) *triCount = vcount;
  return fabs(volume);
}
double or_mt_volume(or_solver* s, double iso, int64_t* triCount) {
  return mt_volume_impl(s->dens, s->nx, s->ny, s->nz, s->dx, iso, triCount, NULL, NULL, 0);
}
double or_mt_volume_field(const void* dens, int nx, int ny, int nz, double dx, double iso, int64_t* triCount) {
  return mt_volume_impl((const st_t*)dens, nx, ny, nz, dx, iso, triCount, NULL, NULL, 0);
}
double or_mt_mesh_field(const void* dens, int nx, int ny, int nz, double dx, double iso, float* pos, float* nrm,
                        int64_t maxVerts, int64_t* vertCount) {
  return mt_volume_impl((const st_t*)dens, nx, ny, nz, dx, iso, vertCount, pos, nrm, maxVerts);
}
/* Metaballs.build's kernel field (js/surface.js:203-284): every liquid
 * particle adds (1 - d^2/R^2)^2 to the corners of its own (m+1)^3 lattice
 * within the kernel radius R; Float32Array accumulation in particle order.
 * Returns m; *mdx, *iso and *R give the lattice spacing, the contour level
 * (metaballIso) and the kernel radius in lattice cells. field holds at least
 * (m+1)^3 floats (pass NULL to get m only). */
static double js_round(double x) { double r = floor(x); return (x - r >= 0.5) ? r + 1 : r; }
int or_metaball_field(int nP, const float* px, const float* py, const float* pz, const uint8_t* fl, int nx, double dx,
                      double spacing, double tension, double detail, float* field, double* mdx_out, double* iso_out,
                      double* R_out) {
  double f = 1;                                           /* js/surface.js:241-244 */
  if (isfinite(detail) && detail > 0) f = detail < 0.5 ? 0.5 : (detail > 1.6 ? 1.6 : detail);
  int m = (int)js_round(nx * f);
  if (m < 6) m = 6;
  double mdx = m == nx ? dx : (nx * dx) / m;
  double t = isfinite(tension) ? tension : 0.5;            /* js/surface.js:211-224 */
  t = t < 0 ? 0 : (t > 1 ? 1 : t);
  double R = (1.6 + 2.2 * t) * spacing / mdx, R2 = R * R;
  if (mdx_out) *mdx_out = mdx;
  if (iso_out) *iso_out = 1.5 * pow((1.6 + 2.2 * t) / 1.6, 1.5);
  if (R_out) *R_out = R;
  if (!field) return m;
  long long len = (long long)(m + 1) * (m + 1) * (m + 1);
  memset(field, 0, sizeof(float) * (size_t)len);
  int rad = (int)ceil(R); if (rad > 3) rad = 3;
  long long sj = m + 1, sk = (long long)(m + 1) * sj;
  for (int p = 0; p < nP; p++) {
    if (fl[p] != 0) continue;
    double gx = px[p] / mdx, gy = py[p] / mdx, gz = pz[p] / mdx;
    /* outside (-8, m + 8) (or NaN) the reference's clamped ranges are empty */
    if (!(gx > -8 && gx < m + 8 && gy > -8 && gy < m + 8 && gz > -8 && gz < m + 8)) continue;
    int i0 = (int)js_round(gx), j0 = (int)js_round(gy), k0 = (int)js_round(gz);
    int ia = i0 - rad > 0 ? i0 - rad : 0, ib = i0 + rad < m ? i0 + rad : m;
    int ja = j0 - rad > 0 ? j0 - rad : 0, jb = j0 + rad < m ? j0 + rad : m;
    int ka = k0 - rad > 0 ? k0 - rad : 0, kb = k0 + rad < m ? k0 + rad : m;
    for (int k = ka; k <= kb; k++) {
      double ez = k - gz, dz2 = ez * ez;
      if (dz2 >= R2) continue;
      for (int j = ja; j <= jb; j++) {
        double ey = j - gy, dy2 = dz2 + ey * ey;
        if (dy2 >= R2) continue;
        long long base = k * sk + j * sj;
        for (int i = ia; i <= ib; i++) {
          double ex = i - gx, d2 = dy2 + ex * ex;
          if (d2 >= R2) continue;
          double u = 1 - d2 / R2;
          field[base + i] = (float)(field[base + i] + u * u);
        }
      }
    }
  }
  return m;
}
/* autotuneIso, js/solver.js:3838-3849 */
double or_autotune_iso(or_solver* s) {
  double Vt = s->S.nP * s->S.particleVolume, lo = 0.3, hi = 3.0;
  for (int it = 0; it < 8; it++) {
    double mid = 0.5 * (lo + hi); int64_t cnt = 0;
    double vol = or_mt_volume(s, mid, &cnt);
    int tooBig = cnt > 900000;
    if (tooBig || vol > Vt) lo = mid; else hi = mid;
  }
  return 0.5 * (lo + hi);
}

/* earthCensus, js/main.js:176-186 */
void or_census(or_solver* s, double out[3]) {
  long nL = 0, nI = 0, nV = 0;
  for (int p = 0; p < s->S.nP; p++) {
    int f = s->pflag[p];
    if (f == 0 || f == 1 || f == 4) nL++; else if (f == 5) nI++; else if (f == 2 || f == 3) nV++;
  }
  double tot = (double)(nL + nI + nV);
  if (tot > 0) { out[0] = nL / tot; out[1] = nI / tot; out[2] = nV / tot; }
  else { out[0] = out[1] = out[2] = 0; }
}

/* kineticEnergy, js/solver.js:3914-3921 */
double or_kinetic_energy(or_solver* s) {
  double e = 0, mp = 1000 * s->S.particleVolume;
  for (int p = 0; p < s->S.nP; p++) {
    double v2 = (double)s->pvx[p] * s->pvx[p] + (double)s->pvy[p] * s->pvy[p] + (double)s->pvz[p] * s->pvz[p];
    e += 0.5 * mp * v2;
  }
  return e;
}

/* dryLandFraction, js/solver.js:3593-3623 */
double or_dry_land_fraction(or_solver* s) {
  if (!s->hasTerr) return 0;
  double cx = s->cx, cy = s->cy, cz = s->cz, dx = s->dx, dv = s->tdv;
  int nx = s->nx, ny = s->ny, nz = s->nz, n = s->tn, N = 1200, dry = 0;
  for (int i = 0; i < N; i++) {
    double a = i * 2.399963, uu = 1 - 2 * (i + 0.5) / N;
    double sq = sqrt(1 - uu * uu);
    double ldx = sq * cos(a), ldy = uu, ldz = sq * sin(a);
    double Rt = -1;
    for (double rr = s->Rhi + dv; rr > s->Rlo - dv; rr -= dv * 0.5) {
      int sx = jtrunc((cx + ldx * rr) / dv), sy = jtrunc((cy + ldy * rr) / dv), sz = jtrunc((cz + ldz * rr) / dv);
      if (sx < 0 || sy < 0 || sz < 0 || sx >= n || sy >= n || sz >= n) continue;
      if (s->tsolid[((size_t)sz * n + sy) * n + sx]) { Rt = rr; break; }
    }
    if (Rt < 0 || Rt <= s->S.oceanR) continue;
    int wet = 0;
    for (int st = 1; st <= 4; st++) {
      double rp = Rt + st * dx * 0.55;
      int ii = jtrunc((cx + ldx * rp) / dx), jj = jtrunc((cy + ldy * rp) / dx), kk = jtrunc((cz + ldz * rp) / dx);
      if (ii < 0 || jj < 0 || kk < 0 || ii >= nx || jj >= ny || kk >= nz) break;
      int ct = s->cellType[((long)kk * ny + jj) * nx + ii];
      if (ct == SOLID) continue;
      if (ct == FLUID) wet = 1;
      break;
    }
    if (!wet) dry++;
  }
  return (double)dry / N;
}

/* applyImpulseSphere / stirAt, js/solver.js:3852-3864, 3895-3908 */
void or_apply_impulse_sphere(or_solver* s, double cx, double cy, double cz, double R,
                             double fx, double fy, double fz) {
  double R2 = R * R;
  for (int p = 0; p < s->S.nP; p++) {
    double ex = s->px[p] - cx, ey = s->py[p] - cy, ez = s->pz[p] - cz;
    double d2 = ex * ex + ey * ey + ez * ez;
    if (d2 > R2) continue;
    double fall = 1 - sqrt(d2) / R;
    s->pvx[p] += fx * fall; s->pvy[p] += fy * fall; s->pvz[p] += fz * fall;
    if (s->pflag[p] != 0) s->pflag[p] = 0;
    s->pcool[p] = 0;
  }
}
void or_stir_at(or_solver* s, double cx, double cy, double cz, double vx, double vy, double vz,
                double R, double dt) {
  double R2 = R * R, k = jmin(1, 14 * dt);
  for (int p = 0; p < s->S.nP; p++) {
    double ex = s->px[p] - cx, ey = s->py[p] - cy, ez = s->pz[p] - cz;
    double d2 = ex * ex + ey * ey + ez * ez;
    if (d2 > R2) continue;
    double fall = 1 - sqrt(d2) / R;
    s->pvx[p] = (st_t)(s->pvx[p] + (vx * 1.25 - s->pvx[p]) * k * fall);
    s->pvy[p] = (st_t)(s->pvy[p] + (vy * 1.25 - s->pvy[p]) * k * fall);
    s->pvz[p] = (st_t)(s->pvz[p] + (vz * 1.25 - s->pvz[p]) * k * fall);
    s->pflag[p] = 0;
  }
}

/* Seeded Gaussian stir kick (no reference counterpart; defined by the
 * 128^3 planet workload): a point on the sea surface in a seeded uniform
 * direction d, a seeded tangent direction t, and for every grid-coupled
 * particle within 3 sigma: v += peak * exp(-|x-c|^2 / (2 sigma^2)) * t.
 * Draw order from stirS: u1, theta (direction), phi (tangent angle). */
void or_stir_gaussian(or_solver* s, double sigma, double peak) {
  uint32_t st = s->S.stirS;
  st = lcg(st); double u1 = st / 4294967296.0 * 2 - 1;
  st = lcg(st); double th = st / 4294967296.0 * 6.283185307179586;
  st = lcg(st); double ph = st / 4294967296.0 * 6.283185307179586;
  s->S.stirS = st;
  double sq = sqrt(1 - u1 * u1);
  double dxn = sq * cos(th), dyn = u1, dzn = sq * sin(th);
  double ax = 0, ay = 1, az = 0;
  if (fabs(dyn) > 0.9) { ax = 1; ay = 0; }
  double e1x = dyn * az - dzn * ay, e1y = dzn * ax - dxn * az, e1z = dxn * ay - dyn * ax;
  double e1l = sqrt(e1x * e1x + e1y * e1y + e1z * e1z);
  e1x /= e1l; e1y /= e1l; e1z /= e1l;
  double e2x = dyn * e1z - dzn * e1y, e2y = dzn * e1x - dxn * e1z, e2z = dxn * e1y - dyn * e1x;
  double cph = cos(ph), sph = sin(ph);
  double tx = cph * e1x + sph * e2x, ty = cph * e1y + sph * e2y, tz = cph * e1z + sph * e2z;
  double R = s->S.oceanR;
  double pcx = s->cx + dxn * R, pcy = s->cy + dyn * R, pcz = s->cz + dzn * R;
  double r2max = 9 * sigma * sigma, inv2s2 = 1 / (2 * sigma * sigma);
  for (int p = 0; p < s->S.nP; p++) {
    if (s->pflag[p] != 0) continue;
    double ex = s->px[p] - pcx, ey = s->py[p] - pcy, ez = s->pz[p] - pcz;
    double d2 = ex * ex + ey * ey + ez * ez;
    if (d2 >= r2max) continue;
    double a = peak * exp(-d2 * inv2s2);
    s->pvx[p] = (st_t)(s->pvx[p] + a * tx);
    s->pvy[p] = (st_t)(s->pvy[p] + a * ty);
    s->pvz[p] = (st_t)(s->pvz[p] + a * tz);
  }
}

/* waveImpulse, js/solver.js:3866-3892 (sphere mode). The reference draws from
 * Math.random(); this restatement draws from the seeded stir stream, in the
 * order the library defines: theta, phi, then one draw per particle in index
 * order, taken whether or not the particle is pushed. */
void or_wave_impulse(or_solver* s, double dvx) {
  uint32_t st = s->S.stirS;
  st = lcg(st); double th = st / 4294967296.0 * M_PI * 2;
  st = lcg(st); double ph = acos(2 * (st / 4294967296.0) - 1);
  double dx = sin(ph) * cos(th), dy = cos(ph), dz = sin(ph) * sin(th);
  double cx = s->cx, cy = s->cy, cz = s->cz;
  for (int p = 0; p < s->S.nP; p++) {
    st = lcg(st);
    double ex = s->px[p] - cx, ey = s->py[p] - cy, ez = s->pz[p] - cz;
    double er = sqrt(ex * ex + ey * ey + ez * ez);
    if (er == 0 || isnan(er)) er = 1e-9;
    double pr = (ex * dx + ey * dy + ez * dz) / er;
    if (pr <= 0) continue;
    double f = pr * pr * pr * (0.7 + st / 4294967296.0 * 0.3);
    s->pvx[p] = (st_t)(s->pvx[p] + ex / er * dvx * f);
    s->pvy[p] = (st_t)(s->pvy[p] + ey / er * dvx * f);
    s->pvz[p] = (st_t)(s->pvz[p] + ez / er * dvx * f);
  }
  s->S.stirS = st;
}

/* oceanPoint, js/solver.js:591-608, drawing u1 and theta of each try from
 * the seeded stir stream instead of Math.random(). */
void or_ocean_point(or_solver* s, double minDepth, double out[3]) {
  double need = minDepth ? minDepth : 0.12;
  double cx = s->cx, cy = s->cy, cz = s->cz, oceanR = s->S.oceanR;
  int found = 0;
  double bestD = -1, best[3] = { 0, 0, 0 };
  int haveBest = 0;
  uint32_t st = s->S.stirS;
  for (int att = 0; att < 64; att++) {
    st = lcg(st); double u1 = st / 4294967296.0 * 2 - 1;
    st = lcg(st); double th = st / 4294967296.0 * 6.2831853;
    double sq = sqrt(1 - u1 * u1);
    double dxn = sq * cos(th), dyn = u1, dzn = sq * sin(th);
    double Rt = or_terrain_radius_at(s, cx + dxn * s->Rhi, cy + dyn * s->Rhi, cz + dzn * s->Rhi);
    double dpt = oceanR - Rt;
    if (dpt > need) {
      double rm = (Rt + oceanR) * 0.5;
      out[0] = cx + dxn * rm; out[1] = cy + dyn * rm; out[2] = cz + dzn * rm;
      found = 1;
      break;
    }
    if (dpt > bestD) {
      bestD = dpt; haveBest = 1;
      best[0] = cx + dxn * (Rt + oceanR) * 0.5; best[1] = cy + dyn * (Rt + oceanR) * 0.5;
      best[2] = cz + dzn * (Rt + oceanR) * 0.5;
    }
  }
  s->S.stirS = st;
  if (found) return;
  if (haveBest) { out[0] = best[0]; out[1] = best[1]; out[2] = best[2]; }
  else { out[0] = cx; out[1] = cy + oceanR; out[2] = cz; }
}
