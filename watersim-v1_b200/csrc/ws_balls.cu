// ws_balls.cu — rigid balls coupled to the fluid (sphere world).
//
// addBall (js/solver.js:3910-3912) keeps up to WS_MAX_BALLS balls, each nine
// doubles: x y z vx vy vz r rho submerged. In every substep:
//   k_ball_raster   the balls become moving solids: SOLID cells with the
//                   ball's velocity in the solid-velocity field
//                   (_rasterizeStatic, :918-938); one block, balls in order
//   k_ball_push     particles are pushed out of the balls, balls in order
//                   per particle (_pushBallsChunk, :1009-1026), after
//                   _markFluidCells and again after advection
//   k_ball_hist     the per-ball 24-bucket histogram of liquid radii in the
//                   2.2r..3.2r shell (_updateBalls, :2357-2408)
//   k_ball_update   one block per ball: waterline, Archimedes cap, drag
//                   against the sampled grid velocity, added mass, clamps,
//                   terrain contact (_ballVsTerrain, :2299-2342, scanned by
//                   the block) and the domain shell (:2409-2530)
//   k_ball_contacts ball-ball collisions in pair order (:2543-2563)
// The ball state stays in device memory, so a substep with balls still runs
// as one graph. FP64 arithmetic in the reference's order (-fmad=false).
#include "ws_internal.cuh"
#include "ws_kernels.cuh"

namespace {

enum { BX, BY, BZ, BVX, BVY, BVZ, BR, BRHO, BSUB, BWORDS };
constexpr int kHist = 24;

__device__ __forceinline__ int floor_clamp(double v, int a, int b) {
  double f = floor(v);
  return f < a ? a : (f > b ? b : (int)f);
}
__device__ __forceinline__ int ceil_clamp(double v, int a, int b) {
  double f = ceil(v);
  return f < a ? a : (f > b ? b : (int)f);
}

__global__ void k_ball_raster(Dims d, uint8_t* __restrict__ type, float* __restrict__ sv, const double* __restrict__ balls,
                              int nb, GridDev g) {
  const long long N = d.nCells;
  for (int n = 0; n < nb; n++) {
    const double* b = balls + n * BWORDS;
    // a non-finite ball covers no cell in the reference (NaN bounds, or an
    // infinite distance in the cell test)
    if (!isfinite(b[BX]) || !isfinite(b[BY]) || !isfinite(b[BZ]) || !isfinite(b[BR])) continue;
    const double r = b[BR], rr = (r + 0.4 * d.dx) * (r + 0.4 * d.dx);
    const int i0 = floor_clamp((b[BX] - r) / d.dx, 1, d.nx - 2), i1 = ceil_clamp((b[BX] + r) / d.dx, 1, d.nx - 2);
    const int j0 = floor_clamp((b[BY] - r) / d.dx, 1, d.ny - 2), j1 = ceil_clamp((b[BY] + r) / d.dx, 1, d.ny - 2);
    const int k0 = floor_clamp((b[BZ] - r) / d.dx, 1, d.nz - 2), k1 = ceil_clamp((b[BZ] + r) / d.dx, 1, d.nz - 2);
    const int ni = i1 - i0 + 1, nj = j1 - j0 + 1, nk = k1 - k0 + 1;
    const long long cells = (ni > 0 && nj > 0 && nk > 0) ? (long long)ni * nj * nk : 0;
    for (long long t = threadIdx.x; t < cells; t += blockDim.x) {
      const int i = i0 + (int)(t % ni), j = j0 + (int)((t / ni) % nj), k = k0 + (int)(t / ((long long)ni * nj));
      const double cx = (i + 0.5) * d.dx - b[BX], cy = (j + 0.5) * d.dx - b[BY], cz = (k + 0.5) * d.dx - b[BZ];
      if (cx * cx + cy * cy + cz * cz <= rr) {
        const long long ci = ((long long)k * d.ny + j) * d.nx + i;
        type[ci] = WS_SOLID;
        sv[ci] = (float)b[BVX]; sv[N + ci] = (float)b[BVY]; sv[2 * N + ci] = (float)b[BVZ];
        seed_cell(g, i, j, k);                        // a moving solid keeps its faces active
      }
    }
    __syncthreads();                                  // a later ball overwrites a shared cell
  }
}

__global__ void k_ball_push(PartsDev P, const double* __restrict__ balls, int nb) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nP) return;
  float px = P.px[p], py = P.py[p], pz = P.pz[p];
  float vx = P.pvx[p], vy = P.pvy[p], vz = P.pvz[p];
  bool moved = false;
  for (int n = 0; n < nb; n++) {
    const double* b = balls + n * BWORDS;
    const double rr = b[BR] + 0.002;
    const double ex = px - b[BX], ey = py - b[BY], ez = pz - b[BZ];
    const double d2 = ex * ex + ey * ey + ez * ez;
    if (!(d2 < rr * rr)) continue;
    double dd = sqrt(d2);
    if (!(dd != 0)) dd = 1e-9;
    const double inv = 1 / dd, nxn = ex * inv, nyn = ey * inv, nzn = ez * inv;
    px = (float)(b[BX] + nxn * rr); py = (float)(b[BY] + nyn * rr); pz = (float)(b[BZ] + nzn * rr);
    const double rvx = vx - b[BVX], rvy = vy - b[BVY], rvz = vz - b[BVZ];
    const double vn = rvx * nxn + rvy * nyn + rvz * nzn;
    if (vn < 0) { vx = (float)(vx - nxn * vn); vy = (float)(vy - nyn * vn); vz = (float)(vz - nzn * vn); }
    moved = true;
  }
  if (moved) { P.px[p] = px; P.py[p] = py; P.pz[p] = pz; P.pvx[p] = vx; P.pvy[p] = vy; P.pvz[p] = vz; }
}

__global__ void k_ball_hist(Dims d, PartsDev P, const double* __restrict__ balls, int nb, double hLo, double hSpan,
                            int* __restrict__ hist, int* __restrict__ histC) {
  __shared__ int sh[WS_MAX_BALLS_DEV * (kHist + 1)];      // per ball: 24 buckets, then the shell count
  for (int i = threadIdx.x; i < nb * (kHist + 1); i += blockDim.x) sh[i] = 0;
  __syncthreads();
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < P.nP && P.pflag[p] == 0) {
    const double ppx = P.px[p], ppy = P.py[p], ppz = P.pz[p];
    const double ldx = ppx - d.cx, ldy = ppy - d.cy, ldz = ppz - d.cz;
    const double level = sqrt(ldx * ldx + ldy * ldy + ldz * ldz);
    for (int q = 0; q < nb; q++) {
      const double* bb = balls + q * BWORDS;
      const double bdx = ppx - bb[BX], bdy = ppy - bb[BY], bdz = ppz - bb[BZ];
      const double dh2 = bdx * bdx + bdy * bdy + bdz * bdz;
      const double r1 = 2.2 * bb[BR], r2 = 3.2 * bb[BR];
      if (dh2 < r1 * r1 || dh2 > r2 * r2) continue;
      const double bf = floor(((level - hLo) / hSpan) * kHist);
      atomicAdd(&sh[q * (kHist + 1) + kHist], 1);
      if (bf != bf) continue;                         // NaN bucket: the reference's store is a no-op
      const int bucket = bf < 0 ? 0 : (bf >= kHist ? kHist - 1 : (int)bf);
      atomicAdd(&sh[q * (kHist + 1) + bucket], 1);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nb * (kHist + 1); i += blockDim.x) {
    const int v = sh[i];
    if (!v) continue;
    const int q = i / (kHist + 1), k = i % (kHist + 1);
    atomicAdd(k == kHist ? &histC[q] : &hist[q * kHist + k], v);
  }
}

// _ballVsTerrain, js/solver.js:2299-2342, by the whole block: the reference
// keeps the first voxel (k, j, i order) whose penetration beats the best so
// far, i.e. the largest penetration, earliest voxel on ties; each thread
// scans a strided share and the block reduces (pen, voxel order) exactly so.
// Called by every thread of the block with the same ball; thread 0 applies.
struct Pen { double pen, nx, ny, nz; long long ord; };
__device__ __forceinline__ bool better(const Pen& a, const Pen& b) {   // a ranks before b
  return a.pen > b.pen || (a.pen == b.pen && a.ord < b.ord);
}
__device__ void ball_vs_terrain(const Dims& d, const TerrainDev& t, double* b) {
  __shared__ Pen red[32];
  const int n = t.n; const double dv = t.dv;
  const double bx = b[BX], by = b[BY], bz = b[BZ], br = b[BR];
  int i0 = (int)((bx - br) / dv), i1 = (int)((bx + br) / dv);
  int j0 = (int)((by - br) / dv), j1 = (int)((by + br) / dv);
  int k0 = (int)((bz - br) / dv), k1 = (int)((bz + br) / dv);
  if (i0 < 0) i0 = 0;
  if (j0 < 0) j0 = 0;
  if (k0 < 0) k0 = 0;
  if (i1 > n - 1) i1 = n - 1;
  if (j1 > n - 1) j1 = n - 1;
  if (k1 > n - 1) k1 = n - 1;
  const int ni = i1 - i0 + 1, nj = j1 - j0 + 1, nk = k1 - k0 + 1;
  const long long cells = (ni > 0 && nj > 0 && nk > 0) ? (long long)ni * nj * nk : 0;
  Pen best{ 0, 0, 0, 0, 0x7fffffffffffffffLL };
  for (long long v = threadIdx.x; v < cells; v += blockDim.x) {     // v ascending = (k, j, i) order
    const int i = i0 + (int)(v % ni), j = j0 + (int)((v / ni) % nj), k = k0 + (int)(v / ((long long)ni * nj));
    if (!t.solid[((long long)k * n + j) * n + i]) continue;
    double qx = bx, qy = by, qz = bz;
    const double vx0 = i * dv, vy0 = j * dv, vz0 = k * dv;
    if (qx < vx0) qx = vx0; else if (qx > vx0 + dv) qx = vx0 + dv;
    if (qy < vy0) qy = vy0; else if (qy > vy0 + dv) qy = vy0 + dv;
    if (qz < vz0) qz = vz0; else if (qz > vz0 + dv) qz = vz0 + dv;
    const double ddx = bx - qx, ddy = by - qy, ddz = bz - qz;
    const double dd = sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
    const double pen = br - dd;
    if (!(pen > best.pen)) continue;
    Pen c{ pen, 0, 0, 0, v };
    if (dd > 1e-6) { c.nx = ddx / dd; c.ny = ddy / dd; c.nz = ddz / dd; }
    else {
      const double rx = bx - d.cx, ry = by - d.cy, rz = bz - d.cz;
      double rl = sqrt(rx * rx + ry * ry + rz * rz);
      if (!(rl != 0)) rl = 1e-9;
      c.nx = rx / rl; c.ny = ry / rl; c.nz = rz / rl;
    }
    best = c;
  }
  for (int o = 16; o > 0; o >>= 1) {
    Pen x;
    x.pen = __shfl_down_sync(0xffffffffu, best.pen, o); x.nx = __shfl_down_sync(0xffffffffu, best.nx, o);
    x.ny = __shfl_down_sync(0xffffffffu, best.ny, o); x.nz = __shfl_down_sync(0xffffffffu, best.nz, o);
    x.ord = __shfl_down_sync(0xffffffffu, best.ord, o);
    if (better(x, best)) best = x;
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  if (lane == 0) red[w] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    Pen bst = red[0];
    for (int q = 1; q < nw; q++) if (better(red[q], bst)) bst = red[q];
    if (bst.pen > 0) {
      b[BX] += bst.nx * (bst.pen + 0.002); b[BY] += bst.ny * (bst.pen + 0.002); b[BZ] += bst.nz * (bst.pen + 0.002);
      const double vn = b[BVX] * bst.nx + b[BVY] * bst.ny + b[BVZ] * bst.nz;
      if (vn < 0) {
        b[BVX] -= bst.nx * vn; b[BVY] -= bst.ny * vn; b[BVZ] -= bst.nz * vn;
        b[BVX] *= 0.985; b[BVY] *= 0.985; b[BVZ] *= 0.985;
      }
    }
  }
  __syncthreads();
}

// _updateBalls forces and integration for one ball, js/solver.js:2434-2502
__device__ void integrate_ball(const Dims& d, const float* __restrict__ vel, double* b, double surf, const BallEnv& env,
                               double dt) {
  const double rhoF = 1000, Cd = 0.5, PI = 3.141592653589793, g = env.gravity;
  const double m = b[BRHO] * 4 / 3 * PI * b[BR] * b[BR] * b[BR];
  const double area = PI * b[BR] * b[BR];
  const double ex0 = b[BX] - d.cx, ey0 = b[BY] - d.cy, ez0 = b[BZ] - d.cz;
  const double bR = sqrt(ex0 * ex0 + ey0 * ey0 + ez0 * ez0);
  const double inner = bR - b[BR];
  double h = surf - inner;
  if (!(h > 0)) h = 0;
  if (h > 2 * b[BR]) h = 2 * b[BR];
  const double Vs = PI * h * h * (3 * b[BR] - h) / 3;
  b[BSUB] = Vs / (4.0 / 3 * PI * b[BR] * b[BR] * b[BR]);
  double upx = 0, upy = 1, upz = 0, gEff = g;
  if (bR > 1e-6) {
    upx = (b[BX] - d.cx) / bR; upy = (b[BY] - d.cy) / bR; upz = (b[BZ] - d.cz) / bR;
    gEff = g * (env.oceanR * env.oceanR) / (bR * bR);
  }
  const double Fb = (rhoF * Vs - m) * gEff;
  double ux, uy, uz;
  sample_vel3(d, vel, b[BX], b[BY], b[BZ], ux, uy, uz);
  const double rvx = b[BVX] - ux, rvy = b[BVY] - uy, rvz = b[BVZ] - uz;
  const double vr = sqrt(rvx * rvx + rvy * rvy + rvz * rvz);
  const double kd = 0.5 * rhoF * Cd * area * vr;
  double Fx = -kd * rvx + upx * Fb, Fz = -kd * rvz + upz * Fb, Fyd = -kd * rvy + upy * Fb;
  const double fdx = Fx - upx * Fb, fdy = Fyd - upy * Fb, fdz = Fz - upz * Fb;
  const double fdm = sqrt(fdx * fdx + fdy * fdy + fdz * fdz);
  const double fdmMax = 0.8 * m * g;
  if (fdm > fdmMax) {
    const double fdc = fdmMax / fdm;
    Fx = upx * Fb + fdx * fdc; Fyd = upy * Fb + fdy * fdc; Fz = upz * Fb + fdz * fdc;
  }
  const double mEff = m + 0.5 * rhoF * Vs;
  b[BVX] += (Fx / mEff) * dt;
  b[BVZ] += (Fz / mEff) * dt;
  b[BVY] += (Fyd / mEff) * dt;
  b[BVX] *= 0.999; b[BVY] *= 0.999; b[BVZ] *= 0.999;
  const double bvmax = 4;
  if (b[BVX] > bvmax) b[BVX] = bvmax; else if (b[BVX] < -bvmax) b[BVX] = -bvmax;
  if (b[BVZ] > bvmax) b[BVZ] = bvmax; else if (b[BVZ] < -bvmax) b[BVZ] = -bvmax;
  if (b[BVY] > bvmax) b[BVY] = bvmax; else if (b[BVY] < -bvmax) b[BVY] = -bvmax;
  b[BX] += b[BVX] * dt; b[BY] += b[BVY] * dt; b[BZ] += b[BVZ] * dt;
}

// the radial constraints after the terrain: the bare core when there is no
// terrain, then the domain shell (js/solver.js:2507-2530)
__device__ void constrain_ball(const Dims& d, bool hasTerrain, double* b, const BallEnv& env) {
  if (!hasTerrain) {
    const double cbx = b[BX] - d.cx, cby = b[BY] - d.cy, cbz = b[BZ] - d.cz;
    double cbr = sqrt(cbx * cbx + cby * cby + cbz * cbz);
    if (!(cbr != 0)) cbr = 1e-9;
    if (cbr < env.coreR + b[BR]) {
      const double rnx0 = cbx / cbr, rny0 = cby / cbr, rnz0 = cbz / cbr, rr0 = env.coreR + b[BR];
      b[BX] = d.cx + rnx0 * rr0; b[BY] = d.cy + rny0 * rr0; b[BZ] = d.cz + rnz0 * rr0;
      const double vn0 = b[BVX] * rnx0 + b[BVY] * rny0 + b[BVZ] * rnz0;
      if (vn0 < 0) {
        b[BVX] -= rnx0 * vn0 * 1.3; b[BVY] -= rny0 * vn0 * 1.3; b[BVZ] -= rnz0 * vn0 * 1.3;
        b[BVX] *= 0.98; b[BVY] *= 0.98; b[BVZ] *= 0.98;
      }
    }
  }
  const double sbx = b[BX] - d.cx, sby = b[BY] - d.cy, sbz = b[BZ] - d.cz;
  double sbr = sqrt(sbx * sbx + sby * sby + sbz * sbz);
  if (!(sbr != 0)) sbr = 1e-9;
  const double rnx = sbx / sbr, rny = sby / sbr, rnz = sbz / sbr;
  if (sbr > d.domainR - b[BR]) {
    const double rr1 = d.domainR - b[BR];
    b[BX] = d.cx + rnx * rr1; b[BY] = d.cy + rny * rr1; b[BZ] = d.cz + rnz * rr1;
    const double vn1 = b[BVX] * rnx + b[BVY] * rny + b[BVZ] * rnz;
    if (vn1 > 0) { b[BVX] -= rnx * vn1 * 1.3; b[BVY] -= rny * vn1 * 1.3; b[BVZ] -= rnz * vn1 * 1.3; }
  }
}

// ball-ball contacts, js/solver.js:2543-2563
__device__ void ball_contacts(double* __restrict__ balls, int nb) {
  for (int a = 0; a < nb; a++) for (int c = a + 1; c < nb; c++) {
    double* A = balls + a * BWORDS;
    double* B = balls + c * BWORDS;
    const double ex = B[BX] - A[BX], ey = B[BY] - A[BY], ez = B[BZ] - A[BZ];
    const double d2 = ex * ex + ey * ey + ez * ez, rSum = A[BR] + B[BR];
    if (d2 > rSum * rSum || d2 < 1e-12) continue;
    const double dd = sqrt(d2), nxn = ex / dd, nyn = ey / dd, nzn = ez / dd;
    const double overlap = rSum - dd;
    const double mA = A[BRHO] * A[BR] * A[BR] * A[BR], mB = B[BRHO] * B[BR] * B[BR] * B[BR];
    const double tA = mB / (mA + mB), tB = mA / (mA + mB);
    A[BX] -= nxn * overlap * tA; A[BY] -= nyn * overlap * tA; A[BZ] -= nzn * overlap * tA;
    B[BX] += nxn * overlap * tB; B[BY] += nyn * overlap * tB; B[BZ] += nzn * overlap * tB;
    const double rvn = (B[BVX] - A[BVX]) * nxn + (B[BVY] - A[BVY]) * nyn + (B[BVZ] - A[BVZ]) * nzn;
    if (rvn < 0) {
      const double jimp = -(1 + 0.3) * rvn / (1 / mA + 1 / mB);
      A[BVX] -= nxn * jimp / mA; A[BVY] -= nyn * jimp / mA; A[BVZ] -= nzn * jimp / mA;
      B[BVX] += nxn * jimp / mB; B[BVY] += nyn * jimp / mB; B[BVZ] += nzn * jimp / mB;
    }
  }
}

// _updateBalls after the histogram, js/solver.js:2409-2530 (sphere world),
// one block per ball (the balls are independent until their contacts): the
// waterline from the ball's histogram (cleared for the next substep), forces
// and integration by thread 0 on a shared copy, the terrain scan by the
// block, then the radial constraints
__global__ void k_ball_update(Dims d, const float* __restrict__ vel, TerrainDev t, double* __restrict__ balls,
                              int* __restrict__ hist, int* __restrict__ histC, float* __restrict__ surfY, BallEnv env,
                              double dt) {
  __shared__ int h[kHist + 1];
  __shared__ double sb[BWORDS];
  const int q = blockIdx.x;
  if (threadIdx.x < kHist) { h[threadIdx.x] = hist[q * kHist + threadIdx.x]; hist[q * kHist + threadIdx.x] = 0; }
  if (threadIdx.x == kHist) { h[kHist] = histC[q]; histC[q] = 0; }
  if (threadIdx.x < BWORDS) sb[threadIdx.x] = balls[q * BWORDS + threadIdx.x];
  __syncthreads();
  if (threadIdx.x == 0) {
    const double hLo = env.coreR, hSpan = (env.oceanR - env.coreR) * 1.5;
    const int total = h[kHist];
    double wl = -INFINITY;
    if (total > 20) {                                   // js/solver.js:2409-2431
      double acc = 0;
      const double target = total * 0.10;
      for (int bkt = kHist - 1; bkt >= 0; bkt--) {
        acc += (float)h[bkt];
        if (acc >= target) { wl = hLo + (bkt + 0.5) / kHist * hSpan; break; }
      }
      if (wl == -INFINITY || total < 140) wl = env.oceanR;
      const double wlMax = env.oceanR + (env.oceanR - env.coreR) * 0.3;
      if (wl > wlMax) wl = wlMax;
      if (wl < env.coreR) wl = env.coreR;
    } else {
      wl = env.oceanR;
    }
    const float surf = (float)wl;                       // the reference keeps it in a Float32Array
    surfY[q] = surf;
    integrate_ball(d, vel, sb, surf, env, dt);
  }
  __syncthreads();
  if (t.has) ball_vs_terrain(d, t, sb);
  if (threadIdx.x == 0) constrain_ball(d, t.has, sb, env);
  __syncthreads();
  if (threadIdx.x < BWORDS) balls[q * BWORDS + threadIdx.x] = sb[threadIdx.x];
}

// the ball-ball contacts, in pair order on a shared copy of all balls
__global__ void k_ball_contacts(double* __restrict__ balls, int nb) {
  __shared__ double sb[WS_MAX_BALLS_DEV * BWORDS];
  for (int i = threadIdx.x; i < nb * BWORDS; i += blockDim.x) sb[i] = balls[i];
  __syncthreads();
  if (threadIdx.x == 0) ball_contacts(sb, nb);
  __syncthreads();
  for (int i = threadIdx.x; i < nb * BWORDS; i += blockDim.x) balls[i] = sb[i];
}

}  // namespace

void launch_ball_raster(const Dims& d, uint8_t* type, float* sv, bool clearSv, const double* balls, int nb,
                        const GridDev& g, cudaStream_t s) {
  if (clearSv) cudaMemsetAsync(sv, 0, sizeof(float) * 3 * (size_t)d.nCells, s);
  if (nb > 0) k_ball_raster<<<1, 256, 0, s>>>(d, type, sv, balls, nb, g);
}
void launch_ball_push(const PartsDev& P, const double* balls, int nb, cudaStream_t s) {
  if (nb > 0 && P.nP > 0) k_ball_push<<<grid_for(P.nP, 256), 256, 0, s>>>(P, balls, nb);
}
void launch_ball_update(const Dims& d, const float* vel, const TerrainDev& t, const PartsDev& P, double* balls, int nb,
                        int* hist, float* surfY, const BallEnv& env, double dt, cudaStream_t s) {
  if (nb <= 0) return;
  int* histC = hist + WS_MAX_BALLS_DEV * kHist;
  if (P.nP > 0)
    k_ball_hist<<<grid_for(P.nP, 256), 256, 0, s>>>(d, P, balls, nb, env.coreR, (env.oceanR - env.coreR) * 1.5, hist,
                                                     histC);
  k_ball_update<<<nb, 128, 0, s>>>(d, vel, t, balls, hist, histC, surfY, env, dt);
  if (nb > 1) k_ball_contacts<<<1, 128, 0, s>>>(balls, nb);
}
