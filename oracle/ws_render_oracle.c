/*
 * ws_render_oracle.c — TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of WaterScene.updateParticles (js/scene.js:1595-1922): the
 * per-class particle staging (liquid beads, spray/rain, vapour, cloud, snow),
 * the colours (sun exposure, temperature tint, spin cues, spin-velocity
 * colour mode), the 64-bucket far-to-near counting sort of the squared
 * camera distance, and the sorted draw list (position, colour, alpha, size,
 * sprite tile). Float32 stores at the reference's Float32Array points,
 * double arithmetic elsewhere. It checks ws_render_particles; only tests/
 * load it.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* same layout as ws_render_opts (include/watersim.h) */
typedef struct {
  int32_t show, beadsMode, metaballMode, spinColor, cloudSprite, planetLit, sortOn, useLight, useDepth, useTemp;
  double waterOpa, pOpa, wScale;
  double waterColor[3], sunDir[3], cam[3];
} or_render_opts;

/* js/scene.js:1595-1922; (cx, cy, cz) = the box centre (scene W/2, H/2, D/2),
 * spacing = solver.spacing, spinOn = solver.spinOn */
int64_t or_render_particles(const or_render_opts* o, double cx, double cy, double cz, double spacing, int spinOn,
                            int n, const float* px, const float* py, const float* pz,
                            const uint8_t* fl, const float* T, const float* pLight, const uint8_t* pDepth,
                            const float* pPh, const float* pWx, const float* pWy, const float* pWz,
                            float* allPos, float* allCol, float* allAlpha, float* allSize, float* allSprite,
                            int32_t counts[5]) {
  /* class staging (Float32Array) */
  float *cPos[5], *cCol[5];
  for (int c = 0; c < 5; c++) { cPos[c] = malloc(sizeof(float) * 3 * (n ? n : 1)); cCol[c] = malloc(sizeof(float) * 3 * (n ? n : 1)); }
  int cnt[5] = { 0, 0, 0, 0, 0 };   /* 0 beads, 1 spray, 2 vapour, 3 cloud, 4 snow */
  /* js/scene.js:1601-1602 */
  int showBeads = o->show && o->beadsMode && o->waterOpa > 0.01 && !o->metaballMode;
  int showSpray = o->show && o->pOpa > 0.01;
  int hasLight = o->useLight, hasDepth = o->useDepth, hasT = o->useTemp, spinCue = spinOn;
  for (int c = 0; c < 5; c++) counts[c] = 0;
  if (!(showBeads || showSpray)) { for (int c = 0; c < 5; c++) { free(cPos[c]); free(cCol[c]); } return 0; }
  int spinCol = o->spinColor != 0;
  double wRx = 0, wRy = 0, wRz = 0, wMx = 0, wMy = 0, wMz = 0;
  if (spinCol) {
    double loX = INFINITY, loY = INFINITY, loZ = INFINITY, hiX = -INFINITY, hiY = -INFINITY, hiZ = -INFINITY;
    for (int q = 0; q < n; q++) {
      double a = pWx[q], b = pWy[q], c = pWz[q];
      if (a < loX) loX = a;
      if (a > hiX) hiX = a;
      if (b < loY) loY = b;
      if (b > hiY) hiY = b;
      if (c < loZ) loZ = c;
      if (c > hiZ) hiZ = c;
    }
    wMx = loX; wMy = loY; wMz = loZ;
    wRx = hiX > loX ? 1 / (hiX - loX) : 0; wRy = hiY > loY ? 1 / (hiY - loY) : 0; wRz = hiZ > loZ ? 1 / (hiZ - loZ) : 0;
  }
  const double pcx = cx, pcy = cy, pcz = cz;
  const double sdx = o->sunDir[0], sdy = o->sunDir[1], sdz = o->sunDir[2], sln = 1;
  for (int p = 0; p < n; p++) {
    double expo = 1;
    if (o->planetLit) {
      if (hasLight) {
        expo = pLight[p];
        if (!(expo > 0)) expo = 0; else if (expo > 1) expo = 1;
      } else {
        double exn = px[p] - pcx, eyn = py[p] - pcy, ezn = pz[p] - pcz;
        double eln = sqrt(exn * exn + eyn * eyn + ezn * ezn); if (!(eln > 0)) eln = 1e-6;
        expo = (exn * sdx + eyn * sdy + ezn * sdz) / (eln * sln);
        if (expo < 0) expo = 0;
      }
    }
    double br = 0.12 + 0.88 * expo;
    int sunnyBead = 0;
    double sR = 0.5, sG = 0.5, sB = 0.5;
    if (spinCol) {
      sR = wRx ? (pWx[p] - wMx) * wRx : 0.5;
      sG = wRy ? (pWy[p] - wMy) * wRy : 0.5;
      sB = wRz ? (pWz[p] - wMz) * wRz : 0.5;
    }
    int f = fl[p], c, i3;
    if (f == 3) {
      if (!showSpray) continue;
      c = 3; i3 = cnt[c]++ * 3;
      cPos[c][i3] = px[p]; cPos[c][i3 + 1] = py[p]; cPos[c][i3 + 2] = pz[p];
      if (spinCol) { cCol[c][i3] = (float)sR; cCol[c][i3 + 1] = (float)sG; cCol[c][i3 + 2] = (float)sB; }
      else {
        double cl = 0.30 + 0.70 * br;
        if (spinCue) cl *= 0.9 + 0.1 * cos(pPh[p]);
        cCol[c][i3] = (float)(0.88 * cl); cCol[c][i3 + 1] = (float)(0.90 * cl); cCol[c][i3 + 2] = (float)(0.93 * cl);
      }
      continue;
    }
    if (f == 5) {
      if (!showSpray) continue;
      c = 4; i3 = cnt[c]++ * 3;
      cPos[c][i3] = px[p]; cPos[c][i3 + 1] = py[p]; cPos[c][i3 + 2] = pz[p];
      if (spinCol) { cCol[c][i3] = (float)sR; cCol[c][i3 + 1] = (float)sG; cCol[c][i3 + 2] = (float)sB; }
      else { double sw = 0.62 + 0.38 * br; cCol[c][i3] = (float)sw; cCol[c][i3 + 1] = (float)sw; cCol[c][i3 + 2] = (float)sw; }
      continue;
    }
    if (f == 2) {
      if (!showSpray) continue;
      c = 2; i3 = cnt[c]++ * 3;
      cPos[c][i3] = px[p]; cPos[c][i3 + 1] = py[p]; cPos[c][i3 + 2] = pz[p];
      if (spinCol) { cCol[c][i3] = (float)sR; cCol[c][i3 + 1] = (float)sG; cCol[c][i3 + 2] = (float)sB; }
      else {
        double cloudLight = 0.22 + 0.78 * br;
        if (spinCue) cloudLight *= 0.85 + 0.15 * cos(pPh[p]);
        cCol[c][i3] = (float)(0.76 * cloudLight); cCol[c][i3 + 1] = (float)(0.85 * cloudLight); cCol[c][i3 + 2] = (float)cloudLight;
      }
      continue;
    }
    if (f == 0) {
      if (!showBeads) continue;
      int sunny = !o->planetLit;
      if (!sunny) {
        double sx0 = px[p] - pcx, sy0 = py[p] - pcy, sz0 = pz[p] - pcz;
        double sl0 = sqrt(sx0 * sx0 + sy0 * sy0 + sz0 * sz0); if (!(sl0 > 0)) sl0 = 1e-6;
        sunny = (sx0 * sdx + sy0 * sdy + sz0 * sdz) / (sl0 * sln) > 0;
      }
      if (!sunny && hasDepth && pDepth[p] > 1) continue;
      sunnyBead = sunny;
      c = 0;
    } else {
      if (!showSpray) continue;
      c = 1;
    }
    i3 = cnt[c]++ * 3;
    cPos[c][i3] = px[p]; cPos[c][i3 + 1] = py[p]; cPos[c][i3 + 2] = pz[p];
    double t = hasT ? T[p] : 0.32; if (t < 0) t = 0; else if (t > 1) t = 1;
    double w = pow(t, 1.4);
    double cr = o->waterColor[0] * (0.9 + 0.1 * w), cg = o->waterColor[1], cb = o->waterColor[2];
    if (f == 1 || f == 4) { cr = cr * 0.45 + 0.55; cg = cg * 0.45 + 0.55; cb = cb * 0.45 + 0.55; }
    if (f == 0) {
      if (spinCol) { cCol[c][i3] = (float)sR; cCol[c][i3 + 1] = (float)sG; cCol[c][i3 + 2] = (float)sB; }
      else { double brr = sunnyBead ? 1 : br; cCol[c][i3] = (float)(cr * brr); cCol[c][i3 + 1] = (float)(cg * brr); cCol[c][i3 + 2] = (float)(cb * brr); }
    } else {
      if (spinCol) { cCol[c][i3] = (float)sR; cCol[c][i3 + 1] = (float)sG; cCol[c][i3 + 2] = (float)sB; }
      else { cCol[c][i3] = (float)(cr * br); cCol[c][i3 + 1] = (float)(cg * br); cCol[c][i3 + 2] = (float)(cb * br); }
    }
  }
  for (int c = 0; c < 5; c++) counts[c] = cnt[c];
  int total = cnt[0] + cnt[1] + cnt[2] + cnt[3] + cnt[4];
  if (!total) { for (int c = 0; c < 5; c++) { free(cPos[c]); free(cCol[c]); } return 0; }
  double spSz = spacing; if (!(isfinite(spSz) && spSz > 0.02)) spSz = 0.06;
  double wS = o->wScale ? o->wScale : 1;
  double sz[5], al[5], sp[5];
  sz[0] = spSz * 3.4; sz[1] = spSz * 3.4 / 3;
  sz[2] = fmax(0.18 * wS, fmin(0.4 * wS, spSz * 5)); sz[3] = fmax(0.30 * wS, fmin(0.62 * wS, spSz * 6.5)); sz[4] = spSz * 3.4;
  al[0] = fmin(1, fmax(0, o->waterOpa)); al[1] = fmin(1, 0.95 * o->pOpa); al[2] = 0.23 * sqrt(o->pOpa);
  al[3] = fmin(1, 0.88 * o->pOpa); al[4] = 1;
  sp[0] = 0; sp[1] = 1; sp[2] = 2; sp[4] = 4;
  sp[3] = o->cloudSprite ? 5 : 3;                    /* CLOUD_SPRITE_TILE = 5 */
  int off[5]; off[0] = 0; for (int c = 1; c < 5; c++) off[c] = off[c - 1] + cnt[c - 1];
  /* element e -> (class, index) in the concatenated order beads, spray, vapour, cloud, snow */
  /* camera in the planet frame, or the centre when there is none (js/scene.js:1807-1817) */
  const double clx = o->sortOn ? o->cam[0] : pcx, cly = o->sortOn ? o->cam[1] : pcy, clz = o->sortOn ? o->cam[2] : pcz;
  float* d2 = malloc(sizeof(float) * total);
  uint32_t* ord = malloc(sizeof(uint32_t) * total);
  for (int c = 0; c < 5; c++)
    for (int e = 0; e < cnt[c]; e++) {
      double dx2 = cPos[c][e * 3] - clx, dy2 = cPos[c][e * 3 + 1] - cly, dz2 = cPos[c][e * 3 + 2] - clz;
      d2[off[c] + e] = (float)(dx2 * dx2 + dy2 * dy2 + dz2 * dz2);
    }
  if (o->sortOn && total > 1) {
    double lo = INFINITY, hi = -INFINITY;
    for (int e = 0; e < total; e++) { double v = d2[e]; if (v < lo) lo = v; if (v > hi) hi = v; }
    const int NB = 64;
    double inv = hi > lo ? (NB - 1) / (hi - lo + 1e-9) : 0;
    int hist[64], bkt[64];
    for (int b = 0; b < NB; b++) hist[b] = 0;
    for (int e = 0; e < total; e++) {
      int bk = (int)((d2[e] - lo) * inv); if (bk < 0) bk = 0; else if (bk >= NB) bk = NB - 1;
      hist[bk]++;
    }
    int acc = 0;
    for (int b = NB - 1; b >= 0; b--) { bkt[b] = acc; acc += hist[b]; }
    for (int e = 0; e < total; e++) {
      int bk = (int)((d2[e] - lo) * inv); if (bk < 0) bk = 0; else if (bk >= NB) bk = NB - 1;
      ord[bkt[bk]++] = (uint32_t)e;
    }
  } else {
    for (int e = 0; e < total; e++) ord[e] = (uint32_t)e;
  }
  for (int k = 0; k < total; k++) {
    int e = (int)ord[k], c = 4;
    while (c > 0 && e < off[c]) c--;
    int i3 = (e - off[c]) * 3;
    for (int d = 0; d < 3; d++) { allPos[k * 3 + d] = cPos[c][i3 + d]; allCol[k * 3 + d] = cCol[c][i3 + d]; }
    allAlpha[k] = (float)al[c]; allSize[k] = (float)sz[c]; allSprite[k] = (float)sp[c];
  }
  free(d2); free(ord);
  for (int c = 0; c < 5; c++) { free(cPos[c]); free(cCol[c]); }
  return total;
}
