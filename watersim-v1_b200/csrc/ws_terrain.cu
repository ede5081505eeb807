// ws_terrain.cu — world setup of the product library: generateTerrain
// (js/solver.js:272-508) and the sphere water fill (_resetWaterSphere,
// :651-731). Setup work, not part of the substep.
//
// Split: the value-noise height field is evaluated per voxel on the GPU in
// FP64 (n^3 independent evaluations); the calibration search, the in-place
// Laplacian smoothing (order-dependent, so kept in the reference's serial
// order), the land-fraction rays and the jittered lattice fill (one serial
// LCG stream) run on the host.
#include "ws_terrain.h"
#include <cmath>
#include <cstring>
#include <vector>

namespace wsterrain {

struct Noise { uint8_t perm[512]; };

static void noise_init(Noise& t, uint32_t seed) {               // js/solver.js:236-245
  uint8_t base[256]; uint32_t s = seed;
  for (int i = 0; i < 256; i++) base[i] = (uint8_t)i;
  for (int i = 255; i > 0; i--) {
    s = s * 1664525u + 1013904223u;
    int j = (int)((s >> 8) % (uint32_t)(i + 1));
    uint8_t tmp = base[i]; base[i] = base[j]; base[j] = tmp;
  }
  for (int i = 0; i < 512; i++) t.perm[i] = base[i & 255];
}

__host__ __device__ inline double nz_h(const uint8_t* perm, int ix, int iy, int iz) {
  return perm[(perm[(perm[ix & 255] + iy) & 255] + iz) & 255] / 255.0;
}
__host__ __device__ inline double nz_fade(double u) { return u * u * u * (u * (u * 6 - 15) + 10); }
__host__ __device__ inline double nz_eval(const uint8_t* perm, double x, double y, double z) {   // :250-261
  double fx = floor(x), fy = floor(y), fz = floor(z);
  int ix = (int)fx, iy = (int)fy, iz = (int)fz;
  double u = nz_fade(x - fx), v = nz_fade(y - fy), w = nz_fade(z - fz);
  double a = nz_h(perm, ix, iy, iz), b = nz_h(perm, ix + 1, iy, iz);
  double c = nz_h(perm, ix, iy + 1, iz), d = nz_h(perm, ix + 1, iy + 1, iz);
  double e = nz_h(perm, ix, iy, iz + 1), f = nz_h(perm, ix + 1, iy, iz + 1);
  double g = nz_h(perm, ix, iy + 1, iz + 1), hh = nz_h(perm, ix + 1, iy + 1, iz + 1);
  double x1 = a + (b - a) * u, x2 = c + (d - c) * u, x3 = e + (f - e) * u, x4 = g + (hh - g) * u;
  double y1 = x1 + (x2 - x1) * v, y2 = x3 + (x4 - x3) * v;
  return y1 + (y2 - y1) * w;
}
__host__ __device__ inline double raw_height(const uint8_t* perm, double bump, double dx, double dy, double dz) {  // :292-313
  double wx = nz_eval(perm, dx * 0.9 + 17.3, dy * 0.9 + 9.1, dz * 0.9 + 4.7) - 0.5;
  double wy = nz_eval(perm, dx * 0.9 + 71.9, dy * 0.9 + 33.7, dz * 0.9 + 21.3) - 0.5;
  double wz = nz_eval(perm, dx * 0.9 + 123.4, dy * 0.9 + 87.2, dz * 0.9 + 55.8) - 0.5;
  double qx = dx + 0.35 * wx, qy = dy + 0.35 * wy, qz = dz + 0.35 * wz;
  double h = 0, amp = 1, fr = 1.15, tot = 0;
  for (int o = 0; o < 4; o++) { h += amp * nz_eval(perm, qx * fr + 3.1, qy * fr + 7.7, qz * fr + 11.9); tot += amp; amp *= 0.5; fr *= 2.1; }
  h /= tot;
  double r = 0; amp = 1; fr = 2.6; tot = 0;
  for (int o = 0; o < 3; o++) {
    double v = nz_eval(perm, qx * fr + 41.2, qy * fr + 23.8, qz * fr + 66.1);
    r += amp * (1 - fabs(2 * v - 1)); tot += amp; amp *= 0.55; fr *= 2.3;
  }
  r /= tot;
  double det = nz_eval(perm, qx * 6.5 + 91.7, qy * 6.5 + 12.4, qz * 6.5 + 78.3);
  return h + 0.45 * bump * (r - 0.5) + 0.14 * bump * (det - 0.5);
}

struct Shape { double Rlo, span, Rsph, mW, cMin, cSpan, offs, bump, cx, cy, cz, dv; int n; };

// voxelisation, js/solver.js:358-372 (terrainR of :342-349 inlined)
__global__ void k_voxelize(Shape S, const uint8_t* __restrict__ permG, float* __restrict__ R) {
  __shared__ uint8_t perm[512];
  for (int i = threadIdx.x; i < 512; i += blockDim.x) perm[i] = permG[i];
  __syncthreads();
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long n = S.n, n3 = n * n * n;
  if (idx >= n3) return;
  int iv = (int)(idx % n), jv = (int)((idx / n) % n), kv = (int)(idx / (n * n));
  double pz0 = (kv + 0.5) * S.dv - S.cz, py0 = (jv + 0.5) * S.dv - S.cy, px0 = (iv + 0.5) * S.dv - S.cx;
  double rr = sqrt(px0 * px0 + py0 * py0 + pz0 * pz0);
  if (rr < 1e-6) { R[idx] = (float)S.Rlo; return; }
  double rv;
  if (S.mW <= 0) rv = S.Rsph;
  else {
    double hv = raw_height(perm, S.bump, px0 / rr, py0 / rr, pz0 / rr);
    double h01 = (hv - S.cMin) / S.cSpan + S.offs;
    if (h01 < 0) h01 = 0; else if (h01 > 1) h01 = 1;
    double rvv = S.Rlo + pow(h01, 1.25) * S.span;
    rv = S.Rsph + (rvv - S.Rsph) * S.mW;
  }
  R[idx] = (float)rv;
}

int generate(const GenInput& in, Terrain& out, std::string& err) {
  double R1 = in.coreR, Rsl = in.seaLevel, bump = in.bumpiness;
  double depthW = std::max(Rsl - R1, 1e-4);
  double Rlo = std::max(R1 * 0.55, Rsl - 1.8889 * depthW);
  double Rhi = Rsl + 0.7778 * depthW;
  double span = Rhi - Rlo;
  double mW = std::min(1.0, bump / 0.3);
  double Rsph = Rsl - std::min(0.4 * depthW, 0.45 * (Rsl - Rlo));
  Noise nf; noise_init(nf, in.seed);
  // calibration over 8192 quasi-uniform directions, :317-341
  const int CALN = 8192;
  std::vector<float> cal(CALN);
  uint32_t cs = in.seed;
  auto crnd = [&cs]() { cs = cs * 1664525u + 1013904223u; return cs / 4294967296.0; };
  double cMin = 1e9, cMax = -1e9;
  for (int ci = 0; ci < CALN; ci++) {
    double u1 = crnd() * 2 - 1; double th = crnd() * 6.2831853;
    double sq = sqrt(1 - u1 * u1);
    double hv = raw_height(nf.perm, bump, sq * cos(th), u1, sq * sin(th));
    cal[ci] = (float)hv;
    if (hv < cMin) cMin = hv; else if (hv > cMax) cMax = hv;
  }
  double cSpan = cMax - cMin; if (cSpan == 0) cSpan = 1;
  double hSl = (Rsl - Rlo) / span, lo = -1, hi = 1, delta = 0;
  for (int it = 0; it < 48; it++) {
    delta = 0.5 * (lo + hi);
    int cnt = 0;
    for (int ci = 0; ci < CALN; ci++) {
      double h01 = (cal[ci] - cMin) / cSpan, hs = h01 + delta;
      if (hs < 0) hs = 0; else if (hs > 1) hs = 1;
      if (pow(hs, 1.25) > hSl) cnt++;
    }
    if (cnt > 0.27 * CALN) hi = delta; else lo = delta;
  }
  double dv = in.dx / 2, W = in.nx * in.dx;
  int n = (int)ceil(W / dv);
  long long n3 = (long long)n * n * n;
  Shape S{Rlo, span, Rsph, mW, cMin, cSpan, delta, bump, in.cx, in.cy, in.cz, dv, n};
  std::vector<float> R((size_t)n3);
  {
    uint8_t* dperm = nullptr; float* dR = nullptr;
    if (cudaMalloc(&dperm, 512) != cudaSuccess || cudaMalloc(&dR, sizeof(float) * n3) != cudaSuccess) {
      cudaFree(dperm); err = "terrain: device allocation failed"; return WS_ERR_NOMEM;
    }
    cudaMemcpyAsync(dperm, nf.perm, 512, cudaMemcpyHostToDevice, in.stream);
    k_voxelize<<<(unsigned)((n3 + 255) / 256), 256, 0, in.stream>>>(S, dperm, dR);
    cudaMemcpyAsync(R.data(), dR, sizeof(float) * n3, cudaMemcpyDeviceToHost, in.stream);
    cudaError_t e = cudaStreamSynchronize(in.stream);
    cudaFree(dperm); cudaFree(dR);
    if (e != cudaSuccess) { err = std::string("terrain: ") + cudaGetErrorString(e); return WS_ERR_CUDA; }
  }
  // slope smoothing in the reference's in-place order, :384-426
  int PASSES = n < 48 ? 1 : (n < 64 ? 2 : 3);
  double BLEND = n < 48 ? 0.15 : (n < 64 ? 0.35 : 0.5);
  long long sN = n, sN2 = (long long)n * n;
  float* Rp = R.data();
  for (int ps = 0; ps < PASSES; ps++) {
    for (long long kv = 1; kv < sN - 1; kv++) {
      long long zB = kv * sN2, zL = (kv - 1) * sN2, zU = (kv + 1) * sN2;
      for (long long jv = 1; jv < sN - 1; jv++) {
        long long yB = zB + jv * sN, yL = zL + (jv - 1) * sN, yU = zL + (jv + 1) * sN;
        long long y2 = zU + (jv - 1) * sN, y3 = zU + jv * sN, y4 = zU + (jv + 1) * sN;
        long long yL2 = zB + (jv - 1) * sN, yU2 = zB + (jv + 1) * sN;
        for (long long iv = 1; iv < sN - 1; iv++) {
          long long iR = yB + iv;
          double avg = ((double)Rp[iR - 1] + Rp[iR + 1] + Rp[yL2 + iv] + Rp[yU2 + iv] +
                        Rp[yL + iv] + Rp[y2 + iv] + Rp[y3 + iv] + Rp[y4 + iv] +
                        Rp[yL + iv - 1] + Rp[yL + iv + 1] + Rp[y2 + iv - 1] + Rp[y2 + iv + 1] +
                        Rp[yU + iv] + Rp[y3 + iv - 1] + Rp[y3 + iv + 1] + Rp[y4 + iv] +
                        Rp[yL2 + iv - 1] + Rp[yL2 + iv + 1]) * (1.0 / 18);
          Rp[iR] = (float)(Rp[iR] + (avg - Rp[iR]) * BLEND);
        }
      }
    }
  }
  double mean0 = 0, mean1 = 0; long long cntR = 0;
  for (long long i = 0; i < n3; i += 7) { mean0 += Rp[i]; cntR++; }
  mean0 /= cntR;
  for (int ps = 0; ps < PASSES; ps++) {
    for (long long kv = 1; kv < sN - 1; kv++) for (long long jv = 1; jv < sN - 1; jv++) {
      long long row = kv * sN2 + jv * sN;
      for (long long iv = 1; iv < sN - 1; iv++) {
        long long iS = row + iv;
        double avg2 = ((double)Rp[iS - 1] + Rp[iS + 1] + Rp[iS - sN] + Rp[iS + sN] + Rp[iS - sN2] + Rp[iS + sN2]) * (1.0 / 6);
        Rp[iS] = (float)(Rp[iS] + (avg2 - Rp[iS]) * BLEND);
      }
    }
  }
  for (long long i = 0; i < n3; i += 7) mean1 += Rp[i];
  mean1 /= cntR;
  if (mean1 > 1e-9) { double sc = mean0 / mean1; for (long long i = 0; i < n3; i++) Rp[i] = (float)(Rp[i] * sc); }
  out.solid.assign((size_t)n3, 0);
  for (long long kv = 0; kv < n; kv++) {
    double pz = (kv + 0.5) * dv - in.cz;
    for (long long jv = 0; jv < n; jv++) {
      double py = (jv + 0.5) * dv - in.cy;
      long long row = (kv * n + jv) * n;
      for (long long iv = 0; iv < n; iv++) {
        double px = (iv + 0.5) * dv - in.cx;
        double rr = sqrt(px * px + py * py + pz * pz);
        out.solid[row + iv] = rr <= Rp[row + iv] ? 1 : 0;
      }
    }
  }
  // land fraction on the voxels, :484-497 (continues the calibration stream)
  int land = 0;
  for (int ci = 0; ci < 4000; ci++) {
    double lu = crnd() * 2 - 1; double lth = crnd() * 6.2831853;
    double lsq = sqrt(1 - lu * lu);
    double ldx = lsq * cos(lth), ldy = lu, ldz = lsq * sin(lth);
    for (double rr2 = Rhi + dv; rr2 > Rlo - dv; rr2 -= dv * 0.5) {
      int sx = (int)((in.cx + ldx * rr2) / dv), sy = (int)((in.cy + ldy * rr2) / dv), sz = (int)((in.cz + ldz * rr2) / dv);
      if (sx < 0 || sy < 0 || sz < 0 || sx >= n || sy >= n || sz >= n) continue;
      if (out.solid[((size_t)sz * n + sy) * n + sx]) { if (rr2 > Rsl) land++; break; }
    }
  }
  out.n = n; out.dv = dv; out.Rsl = Rsl; out.Rlo = Rlo; out.Rhi = Rhi; out.landFrac = land / 4000.0;
  out.R.swap(R);
  return WS_OK;
}

// _rockCellAt through the voxel rule (js/solver.js:553-558) and _voxelRockAt (:565-574)
static inline bool rock_cell(const Terrain& t, const FillInput& in, double x, double y, double z) {
  int i = (int)(x / in.dx), j = (int)(y / in.dx), k = (int)(z / in.dx);
  if (i < 1) i = 1; else if (i > in.nx - 2) i = in.nx - 2;
  if (j < 1) j = 1; else if (j > in.ny - 2) j = in.ny - 2;
  if (k < 1) k = 1; else if (k > in.nz - 2) k = in.nz - 2;
  int vx = (int)((i + 0.5) * in.dx / t.dv), vy = (int)((j + 0.5) * in.dx / t.dv), vz = (int)((k + 0.5) * in.dx / t.dv);
  if (vx < 0) vx = 0; else if (vx >= t.n) vx = t.n - 1;
  if (vy < 0) vy = 0; else if (vy >= t.n) vy = t.n - 1;
  if (vz < 0) vz = 0; else if (vz >= t.n) vz = t.n - 1;
  return t.solid[((size_t)vz * t.n + vy) * t.n + vx] == 1;
}
static inline bool voxel_rock(const Terrain& t, double x, double y, double z) {
  int n = t.n;
  int i = (int)(x / t.dv), j = (int)(y / t.dv), k = (int)(z / t.dv);
  if (i < 0) i = 0; else if (i > n - 1) i = n - 1;
  if (j < 0) j = 0; else if (j > n - 1) j = n - 1;
  if (k < 0) k = 0; else if (k > n - 1) k = n - 1;
  return t.solid[((size_t)k * n + j) * n + i] == 1;
}

double water_volume(const Terrain& t, const FillInput& in) {      // :661-675
  double R2 = in.coreR + in.depth, Rlo = t.Rlo;
  double Vshell = 4.0 / 3 * M_PI * (R2 * R2 * R2 - Rlo * Rlo * Rlo);
  uint32_t mcS = in.seed ^ 0x9e3779b9u; int hits = 0;
  for (int mi = 0; mi < 20000; mi++) {
    mcS = mcS * 1664525u + 1013904223u; double u1 = mcS / 4294967296.0 * 2 - 1;
    mcS = mcS * 1664525u + 1013904223u; double th = mcS / 4294967296.0 * 6.2831853;
    double sq = sqrt(1 - u1 * u1);
    mcS = mcS * 1664525u + 1013904223u;
    double rr = cbrt(Rlo * Rlo * Rlo + mcS / 4294967296.0 * (R2 * R2 * R2 - Rlo * Rlo * Rlo));
    if (!rock_cell(t, in, in.cx + sq * cos(th) * rr, in.cy + u1 * rr, in.cz + sq * sin(th) * rr)) hits++;
  }
  return Vshell * hits / 20000;
}

int fill(const Terrain& t, const FillInput& in, FillOutput& out) {  // :676-718
  double R2 = in.coreR + in.depth;
  double Vw = water_volume(t, in);
  double sp = cbrt(Vw / in.targetParticles);
  double rHi = R2 - 0.4 * sp;
  long long cap = (long long)(in.targetParticles + 8192);
  if (cap > in.capacity) cap = in.capacity;
  out.spacing = sp;
  out.px.clear(); out.py.clear(); out.pz.clear();
  out.px.reserve((size_t)cap); out.py.reserve((size_t)cap); out.pz.reserve((size_t)cap);
  uint32_t fjS = in.seed ^ 0x51ab3c77u;
  long long n = 0;
  for (double y = in.cy - R2; y <= in.cy + R2; y += sp)
    for (double z = in.cz - R2; z <= in.cz + R2; z += sp)
      for (double x = in.cx - R2; x <= in.cx + R2; x += sp) {
        if (n >= cap) break;
        double ex = x - in.cx, ey = y - in.cy, ez = z - in.cz;
        if (ex * ex + ey * ey + ez * ez > rHi * rHi) continue;
        fjS = fjS * 1664525u + 1013904223u; double jx = x + (fjS / 4294967296.0 - 0.5) * sp * 0.3;
        fjS = fjS * 1664525u + 1013904223u; double jy = y + (fjS / 4294967296.0 - 0.5) * sp * 0.3;
        fjS = fjS * 1664525u + 1013904223u; double jz = z + (fjS / 4294967296.0 - 0.5) * sp * 0.3;
        if (rock_cell(t, in, jx, jy, jz) || voxel_rock(t, jx, jy, jz)) continue;
        out.px.push_back((float)jx); out.py.push_back((float)jy); out.pz.push_back((float)jz);
        n++;
      }
  out.capUsed = cap;
  return WS_OK;
}

}  // namespace wsterrain
