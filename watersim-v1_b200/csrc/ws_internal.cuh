// ws_internal.cuh — device state and shared device helpers of libwatersim.
//
// Memory layout in HBM (one handle):
//   particles  SoA, float32 px..pPh, uint8 pflag/pcool/pDepth, capacity each;
//              kept in reference index order so the serial RNG streams of
//              the reference (_evS, _cfS, _bfS) are consumed in its order.
//   faces      vel = u | v | w contiguous (F = uN + vN + wN floats); the same
//              for the snapshot velO, the gravity geometry gvel and the P2G
//              accumulator acc (float2 momentum, weight per face).
//              Index formulas of the reference (js/solver.js:88-113):
//              u (k*ny+j)*(nx+1)+i, v (k*(ny+1)+j)*nx+i, w (k*ny+j)*nx+i.
//   cells      cellType u8, q/rhs/pw float32, cell (k*ny+j)*nx+i.
//
// Arithmetic: the particle passes compute in FP32 with explicit fused
// multiply-adds (P2G, the G2P/advection velocities); every value that decides
// a cell type, a particle phase or a position test stays in FP64, as do the
// residual norm and the volume and census reductions. The SOR iterate is
// FP32 with each update accumulated in FP64 (sor_update says why).
// The rest mirrors the reference (JavaScript doubles over Float32Array
// storage) in FP64; the library is built with -fmad=false so that no FP64
// multiply-add is fused behind the code's back (JavaScript never fuses one).
#pragma once
#include <cmath>
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>
#include "../../include/watersim.h"

#define WS_AIR 0
#define WS_FLUID 1
#define WS_SOLID 2

// device error bits latched in DevStatus::err
#define WS_DERR_NAN 1        // a particle with a non-finite position or velocity (P2G, G2P/advection)
#define WS_DERR_RANGE 2      // a particle outside the domain box when a substep starts
#define WS_DERR_TIMEOUT 4    // a bounded device wait ran out

// Division by an invariant divisor for dividends below 2^31: q = n / d as a
// multiply-high and a shift, m = ceil(2^(31 + l) / d) with l = ceil(log2 d)
// (the error n (m - 2^(31+l)/d) / 2^(31+l) stays below 1/d, so the floor is
// exact). Used to turn flat cell and face indices back into (i, j, k).
struct FastDiv { unsigned m; int s; unsigned d; };
inline FastDiv fastdiv_make(unsigned d) {
  FastDiv f{ 0u, 0, d };
  if (d <= 1) return f;
  int l = 0;
  while ((1ull << l) < d) l++;
  f.m = (unsigned)(((1ull << (31 + l)) + d - 1) / d);
  f.s = l - 1;
  return f;
}
__device__ __forceinline__ unsigned fastdiv(unsigned n, const FastDiv& f) {
  return f.d <= 1 ? n : (__umulhi(n, f.m) >> f.s);
}

struct Dims {
  int nx, ny, nz;
  double dx, W, H, D, cx, cy, cz, domainR;
  long long nCells, uN, vN, wN, F;
  FastDiv dnx, dnx1, dny, dny1;   // nx, nx + 1, ny, ny + 1
  double rdx; int dxPow2;         // 1 / dx, and whether dx is a power of two
};
// A power-of-two divisor b = 2^k: a / b and a * 2^-k are both the correctly
// rounded value of the same real number, so the product is bit-identical to
// the quotient (subnormal and overflowing results included).
inline bool is_pow2(double b) { int e; return b > 0 && std::frexp(b, &e) == 0.5; }
inline void dims_fastdiv(Dims& d) {
  d.dnx = fastdiv_make((unsigned)d.nx); d.dnx1 = fastdiv_make((unsigned)d.nx + 1);
  d.dny = fastdiv_make((unsigned)d.ny); d.dny1 = fastdiv_make((unsigned)d.ny + 1);
  d.dxPow2 = is_pow2(d.dx) ? 1 : 0; d.rdx = 1.0 / d.dx;
}
// (i, j, k) of flat cell index c (c < 2^32) by the invariant-divisor multiply
__device__ __forceinline__ void cell_ijk(const Dims& d, long long c64, int& i, int& j, int& k) {
  const unsigned c = (unsigned)c64, t = fastdiv(c, d.dnx), kk = fastdiv(t, d.dny);
  i = (int)(c - t * (unsigned)d.nx); j = (int)(t - kk * (unsigned)d.ny); k = (int)kk;
}
// v / dx, exactly as the division rounds
__device__ __forceinline__ double over_dx(const Dims& d, double v) { return d.dxPow2 ? v * d.rdx : v / d.dx; }

struct TerrainDev {
  int n, has;
  double dv, Rsl, Rlo, Rhi, Rlo2, Rhi2;
  double rdv; int dvPow2;         // 1 / dv and whether dv is a power of two (see is_pow2)
  const uint8_t* __restrict__ solid;
  const float* __restrict__ R;
};
__device__ __forceinline__ double over_dv(const TerrainDev& t, double v) { return t.dvPow2 ? v * t.rdv : v / t.dv; }

struct PartsDev {
  float *px, *py, *pz, *pvx, *pvy, *pvz, *pT, *pAir, *pLight, *pWx, *pWy, *pWz, *pPh;
  uint8_t *pflag, *pcool, *pDepth;
  int nP;
};

// balls (addBall): capacity, and the scalars _updateBalls reads
#define WS_MAX_BALLS_DEV 64
struct BallEnv { double coreR, oceanR, gravity; };

// render-side particle prep (WaterScene.updateParticles): the scene state
// resolved on the host, per-class alpha/size/sprite already float
struct RenderCfg {
  int showBeads, showSpray, planetLit, useLight, useDepth, useTemp, spinCue, spinCol, sortOn;
  double center[3], sun[3], cam[3], water[3];
  float alpha[5], size[5], sprite[5];
};
// sorted draw list, device buffers of capacity points
struct RenderOut { float *pos, *col, *alpha, *size, *sprite; };

// subsurface current lattice (stride 4 cells) and its nine waves
// (kx, ky, kz, A, ph per wave, 3 octaves x 3 potential components)
struct CurrField {
  int gnx, gny, gnz;
  double sx;
  float *cfx, *cfy, *cfz;
  const double* w;          // device, 45 doubles
  double drift[3];
};

// per-substep device counters (zeroed by the raster kernel)
struct DevStatus {
  unsigned int umaxBits;   // max |u| as float bits (non-negative floats order as ints)
  int airborne;
  int nFluid;
  int err;
  int vaporCount, nightVapor, evapCount, pad;
  int cfA, bfB;            // draws consumed by the vapour pass (diagnostic)
  int sorIters, pad2;
  double relres;
  double rr, bb;
  unsigned long long evIrr;   // evaporation pass: (ejection << 32 | candidate) of the first irregular kick
  int evNEj, evNC, evKeff;    // ejections in the pass, candidates, tabulated band width
  unsigned int evSEnd, evSStart, pad3;   // stream after the pass; start state of a restarted pass
};

struct GridDev {
  uint8_t* type;
  const uint8_t* staticTypes;
  float* vel;
  float* velO;
  float2* acc;
  uint8_t* valid;
  const float* gvel;
  float *q, *rhs, *pw;
  float *vfx, *vfy, *vfz, *omg, *omx, *omy, *omz;
  float* dens;
  const float* sv;          // solid velocity (3 x nCells: x, y, z) of moving solids, or null
  uint8_t* seed;            // 4^3 bricks holding a particle or a moving solid this substep (or null)
  int nbx, nby;             // bricks per axis (x, y) of the seed map
};
// The 4^3-brick work list of the substep's face and cell passes (ws_grid.cu)
struct BrickSet {
  int nbx, nby, nbz;
  uint8_t* seed;            // bricks holding a particle or moving solid this substep
  uint8_t* act;             // seeds dilated by one brick (kept for the next substep)
  uint8_t* proc;            // this substep's work: act | last substep's act | forced
  int* list;                // the bricks with proc set (in no particular order)
  int* count;
  int* forceAll;            // device flag: process every brick once
  FastDiv dnbx, dnby;       // division by nbx and nby (brick coordinates of a linear brick index)
};
// (bx, by, bz) of linear brick b = (bz * nby + by) * nbx + bx
__device__ __forceinline__ void brick_coords(const BrickSet& B, int b, int& bx, int& by, int& bz) {
  const unsigned r = fastdiv((unsigned)b, B.dnbx), z = fastdiv(r, B.dnby);
  bx = b - (int)(r * (unsigned)B.nbx); by = (int)(r - z * (unsigned)B.nby); bz = (int)z;
}
// Counting sort of the grid-coupled particles by cell, rebuilt every
// substep: P2G then walks each cell's particles in a row. The particle
// arrays themselves stay in index order (the serial random streams of the
// later passes consume them in that order); only the permutation is sorted.
struct CellSort {
  int* count;       // particles per cell key (64 per 4^3 brick, + 1); all zero outside a bin..P2G window
  int* start;       // exclusive prefix sum of count
  int* pcell;       // per particle: the key of the cell it was binned in, or -1
  int* pslot;       // per particle: its rank among that cell's particles
  int* perm;        // particle ids in cell order
  int cap;          // entries of pcell, pslot and perm (the particle capacity)
};

// the seed brick of cell (i, j, k)
__device__ __forceinline__ void seed_cell(const GridDev& g, int i, int j, int k) {
  if (g.seed) g.seed[((k >> 2) * g.nby + (j >> 2)) * g.nbx + (i >> 2)] = 1;
}

// ---------------------------------------------------------------- helpers
// Bounded wait of one thread until *flag >= target (acquire loads at GPU
// scope). After `limit` polls it latches WS_DERR_TIMEOUT and returns false,
// so a peer that never arrives ends the wait with an error, never a hang.
__device__ __forceinline__ bool bounded_wait_geq(const unsigned* flag, unsigned target, long long limit, int* err) {
  long long n = 0;
  for (;;) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(flag) : "memory");
    if (v >= target) return true;
    if (++n > limit) { atomicOr(err, WS_DERR_TIMEOUT); return false; }
  }
}
// Fault latch of a particle a pass reads or writes: a non-finite position or
// velocity latches WS_DERR_NAN; a position outside the box [0, W] x [0, H] x
// [0, D] latches WS_DERR_RANGE (the reference's passes keep particles at
// least 1.02 cells inside it, so only corrupt input gets there). Returns
// whether the particle is sound. Faults are rare: one atomic per faulty particle.
__device__ __forceinline__ bool particle_sound(const Dims& d, double x, double y, double z, double u, double v,
                                               double w, int* err, bool checkRange) {
  if (!(isfinite(x) && isfinite(y) && isfinite(z) && isfinite(u) && isfinite(v) && isfinite(w))) {
    atomicOr(err, WS_DERR_NAN);
    return false;
  }
  if (checkRange && (x < 0 || y < 0 || z < 0 || x > d.W || y > d.H || z > d.D)) atomicOr(err, WS_DERR_RANGE);
  return true;
}
// the same NaN latch on the stored FP32 state (no range check)
__device__ __forceinline__ bool particle_sound_f(float x, float y, float z, float u, float v, float w, int* err) {
  if (!(isfinite(x) && isfinite(y) && isfinite(z) && isfinite(u) && isfinite(v) && isfinite(w))) {
    atomicOr(err, WS_DERR_NAN);
    return false;
  }
  return true;
}
__device__ __forceinline__ int jtrunc(double v) { return (int)v; }
// One red-black SOR update of a fluid cell (js/solver.js:1397-1404):
// q (1 - omega) + (omega / diag) (rhs + the sum of the six neighbour q), with
// q = 0 at the non-fluid neighbours, summed in the order -x, +x, -y, +y, -z,
// +z. q is stored in FP32 and the update is accumulated in FP64 with one
// rounding to FP32, as the reference computes it: an update accumulated in
// FP32 (pairwise sum, one FMA) floors the relative residual of the 128^3
// planet near the 1e-5 tolerance (180 iterations instead of 170 on one
// system, q 6.8e-6 instead of 5.6e-7 from the FP64 solve). Every SOR path
// calls this, so their iterates agree bit for bit.
__device__ __forceinline__ float sor_update(float qc, float pw, float rhs, float n0, float n1, float n2, float n3,
                                            float n4, float n5, double om1) {
  double s = (double)n0;
  s += (double)n1;
  s += (double)n2;
  s += (double)n3;
  s += (double)n4;
  s += (double)n5;
  return (float)((double)qc * om1 + (double)pw * ((double)rhs + s));
}
__device__ __forceinline__ int jfloor_clamp(double v, int a, int b) {
  double f = floor(v);
  if (f < a) return a;
  if (f > b) return b;
  return (int)f;
}
__device__ __forceinline__ double dmin(double a, double b) { return a < b ? a : b; }
__device__ __forceinline__ double dmax(double a, double b) { return a > b ? a : b; }
__host__ __device__ __forceinline__ uint32_t lcg_next(uint32_t s) { return s * 1664525u + 1013904223u; }

// LCG jump-ahead: the affine map s -> a s + c composed k times, by square
// and multiply (mod 2^32 arithmetic is exact in uint32).
__host__ __device__ __forceinline__ uint32_t lcg_jump(uint32_t s, uint32_t k) {
  uint32_t A = 1u, Cc = 0u, a = 1664525u, c = 1013904223u;
  while (k) {
    if (k & 1u) { A = A * a; Cc = Cc * a + c; }
    c = c * (a + 1u); a = a * a;
    k >>= 1;
  }
  return A * s + Cc;
}

// terrainRadiusAt, js/solver.js:512-535
__device__ __forceinline__ double terrain_radius_at(const TerrainDev& t, double coreR, double x, double y, double z) {
  if (!t.has) return coreR;
  int n = t.n; double dv = t.dv;
  double gx, gy, gz;
  if (t.dvPow2) { gx = x * t.rdv - 0.5; gy = y * t.rdv - 0.5; gz = z * t.rdv - 0.5; }
  else { gx = x / dv - 0.5; gy = y / dv - 0.5; gz = z / dv - 0.5; }
  int i = jtrunc(gx), j = jtrunc(gy), k = jtrunc(gz);
  if (i < 0) i = 0; else if (i > n - 2) i = n - 2;
  if (j < 0) j = 0; else if (j > n - 2) j = n - 2;
  if (k < 0) k = 0; else if (k > n - 2) k = n - 2;
  double fx = gx - i, fy = gy - j, fz = gz - k;
  if (fx < 0) fx = 0; else if (fx > 1) fx = 1;
  if (fy < 0) fy = 0; else if (fy > 1) fy = 1;
  if (fz < 0) fz = 0; else if (fz > 1) fz = 1;
  long long b000 = ((long long)k * n + j) * n + i, s7 = (long long)n * n;
  const float* R = t.R;
  double v000 = R[b000], v100 = R[b000 + 1];
  double v010 = R[b000 + n], v110 = R[b000 + n + 1];
  double v001 = R[b000 + s7], v101 = R[b000 + s7 + 1];
  double v011 = R[b000 + s7 + n], v111 = R[b000 + s7 + n + 1];
  double a0 = v000 + (v100 - v000) * fx, a1 = v010 + (v110 - v010) * fx;
  double a2 = v001 + (v101 - v001) * fx, a3 = v011 + (v111 - v011) * fx;
  double b0 = a0 + (a1 - a0) * fy, b1 = a2 + (a3 - a2) * fy;
  return b0 + (b1 - b0) * fz;
}

// _rockCellAt, js/solver.js:542-559: the static cell type at the clamped
// cell equals the voxel at the cell centre (rock) for interior cells.
__device__ __forceinline__ bool rock_cell_at(const Dims& d, const uint8_t* __restrict__ staticTypes,
                                             double x, double y, double z) {
  int i = jtrunc(over_dx(d, x)), j = jtrunc(over_dx(d, y)), k = jtrunc(over_dx(d, z));
  if (i < 1) i = 1; else if (i > d.nx - 2) i = d.nx - 2;
  if (j < 1) j = 1; else if (j > d.ny - 2) j = d.ny - 2;
  if (k < 1) k = 1; else if (k > d.nz - 2) k = d.nz - 2;
  return staticTypes[((long long)k * d.ny + j) * d.nx + i] == WS_SOLID;
}

// Face-grid coordinates of component comp, js/solver.js:737-748
__device__ __forceinline__ void face_coords(const Dims& d, int comp, double x, double y, double z,
                                            int& i0, int& j0, int& k0, double& tx, double& ty, double& tz) {
  double a, b, c;
  const double X = over_dx(d, x), Y = over_dx(d, y), Z = over_dx(d, z);
  if (comp == 0) { a = X; b = Y - 0.5; c = Z - 0.5; }
  else if (comp == 1) { a = X - 0.5; b = Y; c = Z - 0.5; }
  else { a = X - 0.5; b = Y - 0.5; c = Z; }
  double fi = floor(a), fj = floor(b), fk = floor(c);
  if (fi < 0) { i0 = 0; tx = 0; } else if (fi > d.nx - 1) { i0 = d.nx - 1; tx = 1; } else { i0 = (int)fi; tx = a - fi; }
  if (fj < 0) { j0 = 0; ty = 0; } else if (fj > d.ny - 2) { j0 = d.ny - 2; ty = 1; } else { j0 = (int)fj; ty = b - fj; }
  if (fk < 0) { k0 = 0; tz = 0; } else if (fk > d.nz - 2) { k0 = d.nz - 2; tz = 1; } else { k0 = (int)fk; tz = c - fk; }
}
// flat offset into vel (u|v|w) and the j/k strides of component comp
__device__ __forceinline__ void face_strides(const Dims& d, int comp, int i0, int j0, int k0,
                                             long long& idx, long long& sj, long long& sk) {
  int nx = d.nx, ny = d.ny;
  if (comp == 0) { sj = nx + 1; sk = (long long)ny * (nx + 1); idx = ((long long)k0 * ny + j0) * (nx + 1) + i0; }
  else if (comp == 1) { sj = nx; sk = (long long)(ny + 1) * nx; idx = d.uN + ((long long)k0 * (ny + 1) + j0) * nx + i0; }
  else { sj = nx; sk = (long long)ny * nx; idx = d.uN + d.vN + ((long long)k0 * ny + j0) * nx + i0; }
}
__device__ __forceinline__ double tri_sample(const float* __restrict__ a, long long idx, long long sj, long long sk,
                                             double tx, double ty, double tz) {
  double s0 = 1 - tx, s1 = tx, t0 = 1 - ty, t1 = ty, r0 = 1 - tz, r1 = tz;
  long long o1 = idx + sj, o2 = idx + sk, o3 = o2 + sj;
  return (((double)a[idx] * s0 + (double)a[idx + 1] * s1) * t0 + ((double)a[o1] * s0 + (double)a[o1 + 1] * s1) * t1) * r0
       + (((double)a[o2] * s0 + (double)a[o2 + 1] * s1) * t0 + ((double)a[o3] * s0 + (double)a[o3 + 1] * s1) * t1) * r1;
}
// _sampleVel3, js/solver.js:820-854
__device__ __forceinline__ void sample_vel3(const Dims& d, const float* __restrict__ vel, double x, double y, double z,
                                            double& ox, double& oy, double& oz) {
  int i0, j0, k0; double tx, ty, tz; long long idx, sj, sk;
  face_coords(d, 0, x, y, z, i0, j0, k0, tx, ty, tz); face_strides(d, 0, i0, j0, k0, idx, sj, sk);
  ox = tri_sample(vel, idx, sj, sk, tx, ty, tz);
  face_coords(d, 1, x, y, z, i0, j0, k0, tx, ty, tz); face_strides(d, 1, i0, j0, k0, idx, sj, sk);
  oy = tri_sample(vel, idx, sj, sk, tx, ty, tz);
  face_coords(d, 2, x, y, z, i0, j0, k0, tx, ty, tz); face_strides(d, 2, i0, j0, k0, idx, sj, sk);
  oz = tri_sample(vel, idx, sj, sk, tx, ty, tz);
}

// ---- FP32 sampling of the hot particle passes (P2G, G2P, advection)
// Face-grid coordinates of component comp in FP32. With a power-of-two cell
// size (the only kind the reference's planets use) x * (1/dx), the half-cell
// shift, the floor and the fraction are exact in FP32 for positions below
// 2^21 cells, so i0/j0/k0 and tx/ty/tz equal the double computation of
// face_coords bit for bit. Other cell sizes take the double path and round
// the fractions.
__device__ __forceinline__ void face_coords_f(const Dims& d, int comp, float x, float y, float z,
                                              int& i0, int& j0, int& k0, float& tx, float& ty, float& tz) {
  if (!d.dxPow2) {
    double a, b, c;
    face_coords(d, comp, x, y, z, i0, j0, k0, a, b, c);
    tx = (float)a; ty = (float)b; tz = (float)c;
    return;
  }
  const float r = (float)d.rdx;
  const float X = x * r, Y = y * r, Z = z * r;
  const float a = comp == 0 ? X : X - 0.5f, b = comp == 1 ? Y : Y - 0.5f, c = comp == 2 ? Z : Z - 0.5f;
  const float fi = floorf(a), fj = floorf(b), fk = floorf(c);
  if (fi < 0.f) { i0 = 0; tx = 0.f; } else if (fi > (float)(d.nx - 1)) { i0 = d.nx - 1; tx = 1.f; } else { i0 = (int)fi; tx = a - fi; }
  if (fj < 0.f) { j0 = 0; ty = 0.f; } else if (fj > (float)(d.ny - 2)) { j0 = d.ny - 2; ty = 1.f; } else { j0 = (int)fj; ty = b - fj; }
  if (fk < 0.f) { k0 = 0; tz = 0.f; } else if (fk > (float)(d.nz - 2)) { k0 = d.nz - 2; tz = 1.f; } else { k0 = (int)fk; tz = c - fk; }
}
// trilinear blend of the eight faces around idx, FP32 with fused multiply-adds
__device__ __forceinline__ float tri_sample_f(const float* __restrict__ a, long long idx, long long sj, long long sk,
                                              float tx, float ty, float tz) {
  const long long o1 = idx + sj, o2 = idx + sk, o3 = o2 + sj;
  const float a00 = a[idx], a10 = a[idx + 1], a01 = a[o1], a11 = a[o1 + 1];
  const float b00 = a[o2], b10 = a[o2 + 1], b01 = a[o3], b11 = a[o3 + 1];
  const float c0 = fmaf(tx, a10 - a00, a00), c1 = fmaf(tx, a11 - a01, a01);
  const float c2 = fmaf(tx, b10 - b00, b00), c3 = fmaf(tx, b11 - b01, b01);
  const float e0 = fmaf(ty, c1 - c0, c0), e1 = fmaf(ty, c3 - c2, c2);
  return fmaf(tz, e1 - e0, e0);
}
// The stencils of all three components at one position, FP32, with 32-bit
// face offsets (face counts stay below 2^32 for grids up to 1000^3). The
// clamps of face_coords depend only on the axis (i in [0, nx - 1], j in
// [0, ny - 2], k in [0, nz - 2]), and each component takes, per axis, either
// the coordinate or the coordinate less half a cell; so six floors serve the
// nine (index, fraction) pairs, bit for bit those of face_coords_f.
struct Stencil3 {
  unsigned idx[3];              // first face of each component's 2x2x2 stencil
  float tx[3], ty[3], tz[3];
};
__device__ __forceinline__ void axis_floor_frac(float a, int hi, int& i0, float& t) {
  const float f = floorf(a);
  if (f < 0.f) { i0 = 0; t = 0.f; } else if (f > (float)hi) { i0 = hi; t = 1.f; } else { i0 = (int)f; t = a - f; }
}
// j and k strides of component comp, 32-bit
__device__ __forceinline__ void face_strides32(const Dims& d, int comp, unsigned& sj, unsigned& sk) {
  const unsigned nx = (unsigned)d.nx, ny = (unsigned)d.ny;
  if (comp == 0) { sj = nx + 1; sk = ny * (nx + 1); }
  else if (comp == 1) { sj = nx; sk = (ny + 1) * nx; }
  else { sj = nx; sk = ny * nx; }
}
__device__ __forceinline__ void face_stencil3_f(const Dims& d, float x, float y, float z, Stencil3& S) {
  const unsigned nx = (unsigned)d.nx, ny = (unsigned)d.ny, uN = (unsigned)d.uN, vN = (unsigned)d.vN;
  if (!d.dxPow2) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      int i0, j0, k0;
      face_coords_f(d, c, x, y, z, i0, j0, k0, S.tx[c], S.ty[c], S.tz[c]);
      S.idx[c] = c == 0 ? ((unsigned)k0 * ny + (unsigned)j0) * (nx + 1) + (unsigned)i0
               : c == 1 ? uN + ((unsigned)k0 * (ny + 1) + (unsigned)j0) * nx + (unsigned)i0
                        : uN + vN + ((unsigned)k0 * ny + (unsigned)j0) * nx + (unsigned)i0;
    }
    return;
  }
  const float r = (float)d.rdx;
  const float X = x * r, Y = y * r, Z = z * r;
  int iF, iH, jF, jH, kF, kH;
  float txF, txH, tyF, tyH, tzF, tzH;
  axis_floor_frac(X, d.nx - 1, iF, txF); axis_floor_frac(X - 0.5f, d.nx - 1, iH, txH);
  axis_floor_frac(Y, d.ny - 2, jF, tyF); axis_floor_frac(Y - 0.5f, d.ny - 2, jH, tyH);
  axis_floor_frac(Z, d.nz - 2, kF, tzF); axis_floor_frac(Z - 0.5f, d.nz - 2, kH, tzH);
  S.idx[0] = ((unsigned)kH * ny + (unsigned)jH) * (nx + 1) + (unsigned)iF;
  S.tx[0] = txF; S.ty[0] = tyH; S.tz[0] = tzH;
  S.idx[1] = uN + ((unsigned)kH * (ny + 1) + (unsigned)jF) * nx + (unsigned)iH;
  S.tx[1] = txH; S.ty[1] = tyF; S.tz[1] = tzH;
  S.idx[2] = uN + vN + ((unsigned)kF * ny + (unsigned)jH) * nx + (unsigned)iH;
  S.tx[2] = txH; S.ty[2] = tyH; S.tz[2] = tzF;
}
// trilinear blend of component comp's stencil in S (tri_sample_f with 32-bit offsets)
__device__ __forceinline__ float stencil_sample(const Dims& d, const float* __restrict__ a, const Stencil3& S, int comp) {
  unsigned sj, sk;
  face_strides32(d, comp, sj, sk);
  const float* p0 = a + S.idx[comp];
  const float* p1 = p0 + sj;
  const float* p2 = p0 + sk;
  const float* p3 = p2 + sj;
  const float a00 = p0[0], a10 = p0[1], a01 = p1[0], a11 = p1[1];
  const float b00 = p2[0], b10 = p2[1], b01 = p3[0], b11 = p3[1];
  const float tx = S.tx[comp], ty = S.ty[comp], tz = S.tz[comp];
  const float c0 = fmaf(tx, a10 - a00, a00), c1 = fmaf(tx, a11 - a01, a01);
  const float c2 = fmaf(tx, b10 - b00, b00), c3 = fmaf(tx, b11 - b01, b01);
  const float e0 = fmaf(ty, c1 - c0, c0), e1 = fmaf(ty, c3 - c2, c2);
  return fmaf(tz, e1 - e0, e0);
}
// _sampleVel3 (js/solver.js:820-854) in FP32
__device__ __forceinline__ void sample_vel3_f(const Dims& d, const float* __restrict__ vel, float x, float y, float z,
                                              float& ox, float& oy, float& oz) {
  Stencil3 S;
  face_stencil3_f(d, x, y, z, S);
  ox = stencil_sample(d, vel, S, 0);
  oy = stencil_sample(d, vel, S, 1);
  oz = stencil_sample(d, vel, S, 2);
}

// block-wide helpers
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ unsigned warp_max_u(unsigned v) {
  for (int o = 16; o > 0; o >>= 1) { unsigned t = __shfl_down_sync(0xffffffffu, v, o); v = t > v ? t : v; }
  return v;
}

static inline unsigned grid_for(long long n, int block) {
  long long g = (n + block - 1) / block;
  return (unsigned)(g < 1 ? 1 : g);
}
