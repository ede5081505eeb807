// ws_grid.cu — grid-side kernels of the substep (js/solver.js:865-1636, 2629-2653).
//
// Each kernel cites the reference lines it restates. Grid kernels are
// HBM-bound streaming passes; their algorithmic bytes per element are listed
// next to each launcher and used for the roofline report.
#include "ws_kernels.cuh"
#include <algorithm>
#include <cub/cub.cuh>

// ------------------------------------------------------------ face decoding
struct FaceIJK { int comp, i, j, k; long long local; };
// 32-bit index arithmetic: face counts stay below 2^32 for grids up to 1000^3
__device__ __forceinline__ FaceIJK decode_face(const Dims& d, long long f64) {
  FaceIJK r;
  unsigned f = (unsigned)f64, nx = d.nx, ny = d.ny, uN = (unsigned)d.uN, vN = (unsigned)d.vN;
  if (f < uN) {
    r.comp = 0; r.local = f;
    unsigned t = fastdiv(f, d.dnx1); r.i = (int)(f - t * (nx + 1));
    unsigned k = fastdiv(t, d.dny); r.j = (int)(t - k * ny); r.k = (int)k;
  } else if (f < uN + vN) {
    unsigned g = f - uN; r.comp = 1; r.local = g;
    unsigned t = fastdiv(g, d.dnx); r.i = (int)(g - t * nx);
    unsigned k = fastdiv(t, d.dny1); r.j = (int)(t - k * (ny + 1)); r.k = (int)k;
  } else {
    unsigned g = f - uN - vN; r.comp = 2; r.local = g;
    unsigned t = fastdiv(g, d.dnx); r.i = (int)(g - t * nx);
    unsigned k = fastdiv(t, d.dny); r.j = (int)(t - k * ny); r.k = (int)k;
  }
  return r;
}
__device__ __forceinline__ void decode_cell(const Dims& d, long long c64, int& i, int& j, int& k) {
  unsigned c = (unsigned)c64, nx = d.nx, ny = d.ny;
  unsigned t = fastdiv(c, d.dnx); i = (int)(c - t * nx);
  unsigned kk = fastdiv(t, d.dny); j = (int)(t - kk * ny); k = (int)kk;
}
// the two cells a face separates; boundary=true for the domain planes
__device__ __forceinline__ bool face_cells(const Dims& d, const FaceIJK& F, long long& cL, long long& cR) {
  long long nx = d.nx, ny = d.ny;
  if (F.comp == 0) {
    if (F.i == 0 || F.i == d.nx) return true;
    cR = ((long long)F.k * ny + F.j) * nx + F.i; cL = cR - 1;
  } else if (F.comp == 1) {
    if (F.j == 0 || F.j == d.ny) return true;
    cR = ((long long)F.k * ny + F.j) * nx + F.i; cL = cR - nx;
  } else {
    if (F.k == 0 || F.k == d.nz) return true;
    cR = ((long long)F.k * ny + F.j) * nx + F.i; cL = cR - nx * ny;
  }
  return false;
}

// ------------------------------------------------------------ static types
// _rasterizeStatic static part, js/solver.js:872-900: terrain voxel at the
// cell centre, plus the closed domain shell.
__global__ void k_static_types(Dims d, TerrainDev t, double coreR, uint8_t* __restrict__ st) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= d.nCells) return;
  int i, j, k; decode_cell(d, c, i, j, k);
  bool shell = (j == 0 || j == d.ny - 1 || k == 0 || k == d.nz - 1 || i == 0 || i == d.nx - 1);
  bool rock;
  if (t.has) {
    int vx = jtrunc((i + 0.5) * d.dx / t.dv), vy = jtrunc((j + 0.5) * d.dx / t.dv), vz = jtrunc((k + 0.5) * d.dx / t.dv);
    if (vx < 0) vx = 0; else if (vx >= t.n) vx = t.n - 1;
    if (vy < 0) vy = 0; else if (vy >= t.n) vy = t.n - 1;
    if (vz < 0) vz = 0; else if (vz >= t.n) vz = t.n - 1;
    rock = t.solid[((long long)vz * t.n + vy) * t.n + vx] == 1;
  } else {
    double dx2 = (i + 0.5) * d.dx - d.cx, dy2 = (j + 0.5) * d.dx - d.cy, dz2 = (k + 0.5) * d.dx - d.cz;
    rock = dx2 * dx2 + dy2 * dy2 + dz2 * dz2 < coreR * coreR;
  }
  st[c] = (shell || rock) ? WS_SOLID : WS_AIR;
}
void launch_static_types(const Dims& d, const TerrainDev& t, double coreR, uint8_t* st, cudaStream_t s) {
  k_static_types<<<grid_for(d.nCells, 256), 256, 0, s>>>(d, t, coreR, st);
}

// _buildPlanetGravity, js/solver.js:1177-1210: unit-g radial geometry per face
__global__ void k_gravity_geometry(Dims d, double oceanR, float* __restrict__ g) {
  long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (f >= d.F) return;
  FaceIJK F = decode_face(d, f);
  double g0 = oceanR * oceanR, ex, ey, ez, e;
  if (F.comp == 0) { ex = F.i * d.dx - d.cx; ey = (F.j + 0.5) * d.dx - d.cy; ez = (F.k + 0.5) * d.dx - d.cz; e = ex; }
  else if (F.comp == 1) { ex = (F.i + 0.5) * d.dx - d.cx; ey = F.j * d.dx - d.cy; ez = (F.k + 0.5) * d.dx - d.cz; e = ey; }
  else { ex = (F.i + 0.5) * d.dx - d.cx; ey = (F.j + 0.5) * d.dx - d.cy; ez = F.k * d.dx - d.cz; e = ez; }
  double r3 = pow(ex * ex + ey * ey + ez * ez, 1.5);
  if (r3 == 0) r3 = 1e-9;
  g[f] = (float)(-g0 * e / r3);
}
void launch_gravity_geometry(const Dims& d, double oceanR, float* g, cudaStream_t s) {
  k_gravity_geometry<<<grid_for(d.F, 256), 256, 0, s>>>(d, oceanR, g);
}

// ------------------------------------------------------------ 1. clear + raster
// u..wW.fill(0) (js/solver.js:2569-2570) and cellType <- static types
// (:865-871). Bytes: 8F (acc) + 2N.
// 16-byte stores: two faces of the accumulator, sixteen cell types per
// thread (both buffers are separate allocations, 256-byte aligned).
__global__ void k_clear_raster(Dims d, GridDev g, DevStatus* st, int clearAcc) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long F2 = d.F >> 1, n16 = d.nCells >> 4;
  if (clearAcc) {
    if (t < F2) reinterpret_cast<float4*>(g.acc)[t] = make_float4(0.f, 0.f, 0.f, 0.f);
    else if (t == F2 && (d.F & 1)) g.acc[d.F - 1] = make_float2(0.f, 0.f);
  }
  if (t < n16) reinterpret_cast<uint4*>(g.type)[t] = reinterpret_cast<const uint4*>(g.staticTypes)[t];
  else if (t < n16 + (d.nCells & 15)) { const long long c = (n16 << 4) + (t - n16); g.type[c] = g.staticTypes[c]; }
  if (t == 0) { st->umaxBits = 0u; st->airborne = 0; st->nFluid = 0; }
}
void launch_clear_raster(const Dims& d, const GridDev& g, DevStatus* st, bool clearAcc, cudaStream_t s) {
  const long long a = clearAcc ? (d.F >> 1) + 1 : 0, b = (d.nCells >> 4) + 16;
  k_clear_raster<<<grid_for(a > b ? a : b, 256), 256, 0, s>>>(d, g, st, clearAcc ? 1 : 0);
}

// ------------------------------------------------------------ 2. mark fluid
// _markFluidCells, js/solver.js:945-1000 (sphere). Bytes: 13P + N.
// the cell a grid-coupled particle marks, or -1 (not coupled, or it turns airborne: pflag 1)
__device__ __forceinline__ long long mark_cell(const Dims& d, const GridDev& g, PartsDev& P, const TerrainDev& t,
                                               double oceanR, double coreR, int p, int fl, double X, double Y,
                                               double Z) {
  if (fl != 0) return -1;
  double rx = X - d.cx, ry = Y - d.cy, rz = Z - d.cz;
  double radius2 = rx * rx + ry * ry + rz * rz;
  double skyAlt = 2 * d.dx > 0.3 ? 2 * d.dx : 0.3;
  if (radius2 > (oceanR + 0.3) * (oceanR + 0.3) &&
      sqrt(radius2) - terrain_radius_at(t, coreR, X, Y, Z) > skyAlt &&
      !(t.has && rock_cell_at(d, g.staticTypes, X, Y, Z))) {
    P.pflag[p] = 1; return -1;
  }
  int i = jfloor_clamp(over_dx(d, X), 0, d.nx - 1);
  int j = jfloor_clamp(over_dx(d, Y), 0, d.ny - 1);
  int k = jfloor_clamp(over_dx(d, Z), 0, d.nz - 1);
  if (j >= d.ny - 2) {
    if (sqrt(radius2) - terrain_radius_at(t, coreR, X, Y, Z) > 0.3) { P.pflag[p] = 1; return -1; }
  }
  return ((long long)k * d.ny + j) * d.nx + i;
}
// Warp-aggregated increment of count[key] for every lane with key >= 0: the
// lanes holding one key share a single atomic; each gets its own rank. All
// 32 lanes of the warp call it (lanes without work pass -1).
__device__ __forceinline__ int warp_rank_inc(int* count, int key) {
  const unsigned peers = __match_any_sync(0xffffffffu, key);
  const int lane = threadIdx.x & 31, leader = __ffs(peers) - 1;
  int base = 0;
  if (lane == leader && key >= 0) base = atomicAdd(&count[key], __popc(peers));
  base = __shfl_sync(0xffffffffu, base, leader);
  return base + __popc(peers & ((1u << lane) - 1u));
}
// the sort key of cell (i, j, k): its 4^3 brick times 64 plus its place in the brick
__device__ __forceinline__ int brick_key(const GridDev& g, int i, int j, int k) {
  return ((((k >> 2) * g.nby + (j >> 2)) * g.nbx + (i >> 2)) << 6) | ((k & 3) << 4) | ((j & 3) << 2) | (i & 3);
}
// Two particles per thread: both particles' loads, then both cells' type
// loads, then the (idempotent) stores, so the two chains overlap. With a
// cell sort (cs.count set) every particle that P2G will scatter (marked, with
// a finite velocity) is also counted in its cell, and its rank recorded.
__global__ void k_mark_fluid(Dims d, GridDev g, PartsDev P, TerrainDev t, double oceanR, double coreR, CellSort cs,
                             int* err) {
  const int p0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x), p1 = p0 + 1;
  const bool has0 = p0 < P.nP, has1 = p1 < P.nP;
  long long c0 = -1, c1 = -1;
  bool fin0 = false, fin1 = false;
  if (has0) {
    const int fl0 = P.pflag[p0], fl1 = has1 ? P.pflag[p1] : 1;
    const double X0 = P.px[p0], Y0 = P.py[p0], Z0 = P.pz[p0];
    const double X1 = has1 ? P.px[p1] : 0.0, Y1 = has1 ? P.py[p1] : 0.0, Z1 = has1 ? P.pz[p1] : 0.0;
    if (cs.count) {
      fin0 = isfinite(P.pvx[p0]) && isfinite(P.pvy[p0]) && isfinite(P.pvz[p0]);
      fin1 = has1 && isfinite(P.pvx[p1]) && isfinite(P.pvy[p1]) && isfinite(P.pvz[p1]);
    }
    // the first pass of a substep to read the positions: every particle must
    // be finite and inside the domain box (the reference's passes keep it there)
    particle_sound(d, X0, Y0, Z0, 0.0, 0.0, 0.0, err, true);
    if (has1) particle_sound(d, X1, Y1, Z1, 0.0, 0.0, 0.0, err, true);
    // the brick of every particle's cell seeds this substep's active bricks
    seed_cell(g, jfloor_clamp(over_dx(d, X0), 0, d.nx - 1), jfloor_clamp(over_dx(d, Y0), 0, d.ny - 1),
              jfloor_clamp(over_dx(d, Z0), 0, d.nz - 1));
    if (has1)
      seed_cell(g, jfloor_clamp(over_dx(d, X1), 0, d.nx - 1), jfloor_clamp(over_dx(d, Y1), 0, d.ny - 1),
                jfloor_clamp(over_dx(d, Z1), 0, d.nz - 1));
    c0 = mark_cell(d, g, P, t, oceanR, coreR, p0, fl0, X0, Y0, Z0);
    c1 = mark_cell(d, g, P, t, oceanR, coreR, p1, fl1, X1, Y1, Z1);
    const uint8_t t0 = c0 >= 0 ? g.type[c0] : (uint8_t)WS_SOLID, t1 = c1 >= 0 ? g.type[c1] : (uint8_t)WS_SOLID;
    if (t0 == WS_AIR) g.type[c0] = WS_FLUID;
    if (t1 == WS_AIR) g.type[c1] = WS_FLUID;
  }
  if (!cs.count) return;                                // uniform over the launch
  // a marked particle with a non-finite velocity stays off the grid and is latched
  if ((c0 >= 0 && !fin0) || (c1 >= 0 && !fin1)) atomicOr(err, WS_DERR_NAN);
  auto key_of = [&](long long c) { int i, j, k; cell_ijk(d, c, i, j, k); return brick_key(g, i, j, k); };
  const int k0 = c0 >= 0 && fin0 ? key_of(c0) : -1, k1 = c1 >= 0 && fin1 ? key_of(c1) : -1;
  const int r0 = warp_rank_inc(cs.count, k0), r1 = warp_rank_inc(cs.count, k1);
  if (has0) { cs.pcell[p0] = k0; cs.pslot[p0] = r0; }
  if (has1) { cs.pcell[p1] = k1; cs.pslot[p1] = r1; }
}
// Without the cell sort: four consecutive particles per thread (float4 and
// uchar4 loads), the seed brick stored once per run of particles in one
// brick, the cell types of all four loaded before any store, and a store
// once per run of particles in one cell. Same marks as k_mark_fluid.
__global__ void __launch_bounds__(256) k_mark_fluid_runs(Dims d, GridDev g, PartsDev P, TerrainDev t, double oceanR,
                                                         double coreR, int* err) {
  const int p0 = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
  if (p0 >= P.nP) return;
  float xs[4], ys[4], zs[4];
  int fl[4];
  int nHave = 4;
  if (p0 + 3 < P.nP) {                                // the arrays are 16-byte aligned and p0 % 4 == 0
    const float4 X = *reinterpret_cast<const float4*>(P.px + p0), Y = *reinterpret_cast<const float4*>(P.py + p0);
    const float4 Z = *reinterpret_cast<const float4*>(P.pz + p0);
    const uchar4 F = *reinterpret_cast<const uchar4*>(P.pflag + p0);
    xs[0] = X.x; xs[1] = X.y; xs[2] = X.z; xs[3] = X.w; ys[0] = Y.x; ys[1] = Y.y; ys[2] = Y.z; ys[3] = Y.w;
    zs[0] = Z.x; zs[1] = Z.y; zs[2] = Z.z; zs[3] = Z.w; fl[0] = F.x; fl[1] = F.y; fl[2] = F.z; fl[3] = F.w;
  } else {
    nHave = P.nP - p0;
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const bool has = r < nHave;
      xs[r] = has ? P.px[p0 + r] : 0.f; ys[r] = has ? P.py[p0 + r] : 0.f; zs[r] = has ? P.pz[p0 + r] : 0.f;
      fl[r] = has ? P.pflag[p0 + r] : 1;
    }
  }
  long long c[4];
  int lastBrick = -1;
#pragma unroll
  for (int r = 0; r < 4; r++) {
    c[r] = -1;
    if (r >= nHave) continue;
    const double X = xs[r], Y = ys[r], Z = zs[r];
    // the first pass of a substep to read the positions: every particle must
    // be finite and inside the domain box (the reference's passes keep it there)
    particle_sound(d, X, Y, Z, 0.0, 0.0, 0.0, err, true);
    // the brick of every particle's cell seeds this substep's active bricks
    const int i = jfloor_clamp(over_dx(d, X), 0, d.nx - 1), j = jfloor_clamp(over_dx(d, Y), 0, d.ny - 1);
    const int k = jfloor_clamp(over_dx(d, Z), 0, d.nz - 1);
    const int sb = ((k >> 2) * g.nby + (j >> 2)) * g.nbx + (i >> 2);
    if (g.seed && sb != lastBrick) { g.seed[sb] = 1; lastBrick = sb; }
    c[r] = mark_cell(d, g, P, t, oceanR, coreR, p0 + r, fl[r], X, Y, Z);
  }
  uint8_t ty[4];
#pragma unroll
  for (int r = 0; r < 4; r++) ty[r] = c[r] >= 0 ? g.type[c[r]] : (uint8_t)WS_SOLID;
#pragma unroll
  for (int r = 0; r < 4; r++)
    if (ty[r] == WS_AIR && (r == 0 || c[r] != c[r - 1])) g.type[c[r]] = WS_FLUID;
}
void launch_mark_fluid(const Dims& d, const GridDev& g, const PartsDev& P, const TerrainDev& t,
                       double oceanR, double coreR, const CellSort* cs, DevStatus* st, cudaStream_t s) {
  if (P.nP <= 0) return;
  if (!cs) {
    k_mark_fluid_runs<<<grid_for((P.nP + 3) / 4, 256), 256, 0, s>>>(d, g, P, t, oceanR, coreR, &st->err);
    return;
  }
  k_mark_fluid<<<grid_for((P.nP + 1) / 2, 256), 256, 0, s>>>(d, g, P, t, oceanR, coreR, *cs, &st->err);
}

// ------------------------------------------------------------ 3. P2G scatter
// _p2gInto, js/solver.js:1035-1105: trilinear momentum + weight per face,
// one float2 vector atomic per face (momentum, weight). FP32 arithmetic: the
// face indices and fractions are exact (face_coords_f), the weights and
// terms carry FP32 rounding (a few 1e-8 relative against the double sums).
//
// Runs of consecutive particles: each thread scatters four consecutive
// particles (the fill's lattice runs along x about a third of a cell apart,
// so three or four neighbours in index order usually share a stencil). Per
// component, the particles' (momentum, weight) terms are summed in registers
// while their stencils start at the same face, and each run sends one set of
// eight float2 atomics.
template <int COMP>
__device__ __forceinline__ void p2g_run_comp(const Dims& d, float2* __restrict__ acc, const float (&x)[4],
                                             const float (&y)[4], const float (&z)[4], const float (&v)[4],
                                             unsigned okMask) {
  unsigned sj, sk;
  face_strides32(d, COMP, sj, sk);
  const unsigned nx = (unsigned)d.nx, ny = (unsigned)d.ny, uN = (unsigned)d.uN, vN = (unsigned)d.vN;
  float m8[8], w8[8];
  unsigned cur = 0xffffffffu;
#define WS_P2G_FLUSH                                                                         \
  if (cur != 0xffffffffu) {                                                                  \
    float2* p = acc + cur;                                                                   \
    atomicAdd(p, make_float2(m8[0], w8[0]));                                                 \
    atomicAdd(p + 1, make_float2(m8[1], w8[1]));                                             \
    atomicAdd(p + sj, make_float2(m8[2], w8[2]));                                            \
    atomicAdd(p + sj + 1, make_float2(m8[3], w8[3]));                                        \
    atomicAdd(p + sk, make_float2(m8[4], w8[4]));                                            \
    atomicAdd(p + sk + 1, make_float2(m8[5], w8[5]));                                        \
    atomicAdd(p + sk + sj, make_float2(m8[6], w8[6]));                                       \
    atomicAdd(p + sk + sj + 1, make_float2(m8[7], w8[7]));                                   \
  }
#pragma unroll
  for (int r = 0; r < 4; r++) {
    if (!((okMask >> r) & 1u)) continue;
    int i0, j0, k0; float tx, ty, tz;
    face_coords_f(d, COMP, x[r], y[r], z[r], i0, j0, k0, tx, ty, tz);
    const unsigned idx = COMP == 0 ? ((unsigned)k0 * ny + (unsigned)j0) * (nx + 1) + (unsigned)i0
                       : COMP == 1 ? uN + ((unsigned)k0 * (ny + 1) + (unsigned)j0) * nx + (unsigned)i0
                                   : uN + vN + ((unsigned)k0 * ny + (unsigned)j0) * nx + (unsigned)i0;
    const float s0 = 1.f - tx, s1 = tx, t0 = 1.f - ty, t1 = ty, r0 = 1.f - tz, r1 = tz;
    const float wA = s0 * t0, wB = s1 * t0, wC = s0 * t1, wD = s1 * t1;
    const float w[8] = { wA * r0, wB * r0, wC * r0, wD * r0, wA * r1, wB * r1, wC * r1, wD * r1 };
    if (idx != cur) {
      WS_P2G_FLUSH
      cur = idx;
#pragma unroll
      for (int q = 0; q < 8; q++) { m8[q] = w[q] * v[r]; w8[q] = w[q]; }
    } else {
#pragma unroll
      for (int q = 0; q < 8; q++) { m8[q] = fmaf(w[q], v[r], m8[q]); w8[q] += w[q]; }
    }
  }
  WS_P2G_FLUSH
#undef WS_P2G_FLUSH
}
__global__ void __launch_bounds__(256, 4) k_p2g_runs(Dims d, GridDev g, PartsDev P, int* err) {
  const int p0 = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
  if (p0 >= P.nP) return;
  float x[4], y[4], z[4], u[4], v[4], w[4];
  int fl[4];
  if (p0 + 3 < P.nP) {                                // the arrays are 16-byte aligned and p0 % 4 == 0
    const float4 X = *reinterpret_cast<const float4*>(P.px + p0), Y = *reinterpret_cast<const float4*>(P.py + p0);
    const float4 Z = *reinterpret_cast<const float4*>(P.pz + p0), U = *reinterpret_cast<const float4*>(P.pvx + p0);
    const float4 V = *reinterpret_cast<const float4*>(P.pvy + p0), W = *reinterpret_cast<const float4*>(P.pvz + p0);
    const uchar4 F = *reinterpret_cast<const uchar4*>(P.pflag + p0);
    x[0] = X.x; x[1] = X.y; x[2] = X.z; x[3] = X.w; y[0] = Y.x; y[1] = Y.y; y[2] = Y.z; y[3] = Y.w;
    z[0] = Z.x; z[1] = Z.y; z[2] = Z.z; z[3] = Z.w; u[0] = U.x; u[1] = U.y; u[2] = U.z; u[3] = U.w;
    v[0] = V.x; v[1] = V.y; v[2] = V.z; v[3] = V.w; w[0] = W.x; w[1] = W.y; w[2] = W.z; w[3] = W.w;
    fl[0] = F.x; fl[1] = F.y; fl[2] = F.z; fl[3] = F.w;
  } else {
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const int p = p0 + r;
      const bool has = p < P.nP;
      x[r] = has ? P.px[p] : 0.f; y[r] = has ? P.py[p] : 0.f; z[r] = has ? P.pz[p] : 0.f;
      u[r] = has ? P.pvx[p] : 0.f; v[r] = has ? P.pvy[p] : 0.f; w[r] = has ? P.pvz[p] : 0.f;
      fl[r] = has ? P.pflag[p] : 1;
    }
  }
  // a fluid particle with a non-finite state is left out of the grid and latched
  unsigned ok = 0;
#pragma unroll
  for (int r = 0; r < 4; r++)
    if (fl[r] == 0 && particle_sound_f(x[r], y[r], z[r], u[r], v[r], w[r], err)) ok |= 1u << r;
  if (!ok) return;
  p2g_run_comp<0>(d, g.acc, x, y, z, u, ok);
  p2g_run_comp<1>(d, g.acc, x, y, z, v, ok);
  p2g_run_comp<2>(d, g.acc, x, y, z, w, ok);
}
void launch_p2g(const Dims& d, const GridDev& g, const PartsDev& P, DevStatus* st, cudaStream_t s) {
  if (P.nP <= 0) return;
  k_p2g_runs<<<grid_for((P.nP + 3) / 4, 256), 256, 0, s>>>(d, g, P, &st->err);
}

// ------------------------------------------------------------ 3b. P2G in cell order
// The same scatter (_p2gInto, js/solver.js:1035-1105) over the particles
// sorted by cell, brick-major: the key of cell (i, j, k) is its 4^3 brick
// times 64 plus its place in the brick, so a brick's particles are one range
// of the permutation. One block per brick adds every particle's eight FP32
// (momentum, weight) terms per component into a shared-memory copy of the
// faces the brick's particles can reach (red.shared.add.f32), then sends one
// float2 atomic per touched face. Every FP32 term is the one k_p2g_runs adds;
// only the order of the FP32 sums differs. A particle whose stencil leaves
// the brick's faces (a ball pushed it after the binning) adds its terms to
// global memory directly.
static unsigned brick_grid(const BrickSet& B);

// The stage-wise P2G, without a mark pass that counted: the particles P2G
// scatters (pflag 0, finite state) counted per cell, each with its rank.
__global__ void k_bin_cells(Dims d, GridDev g, PartsDev P, CellSort cs, int* err) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  int key = -1;
  if (p < P.nP && P.pflag[p] == 0) {
    const double x = P.px[p], y = P.py[p], z = P.pz[p];
    if (particle_sound(d, x, y, z, P.pvx[p], P.pvy[p], P.pvz[p], err, false))
      key = brick_key(g, jfloor_clamp(over_dx(d, x), 0, d.nx - 1), jfloor_clamp(over_dx(d, y), 0, d.ny - 1),
                      jfloor_clamp(over_dx(d, z), 0, d.nz - 1));
  }
  const int r = warp_rank_inc(cs.count, key);          // every lane of the warp takes part
  if (p < P.nP) { cs.pcell[p] = key; cs.pslot[p] = r; }
}
// particle ids into their cells' ranges
__global__ void k_cell_scatter(int nP, CellSort cs, int* err) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nP) return;
  const int c = cs.pcell[p];
  if (c < 0) return;
  const int at = cs.start[c] + cs.pslot[p];
  if (at >= 0 && at < cs.cap) cs.perm[at] = p;
  else atomicOr(err, WS_DERR_RANGE);
}

// Shared-memory faces of one brick: per component the faces of the brick's
// cells widened by one along the two tangential axes (5 x 6 x 6 = 180), the
// component's own axis keeping its upper face. Momentum sums first, then
// the weights.
constexpr int kBrickFaces = 180;
// origin offset of component comp's face box from the brick's first cell, and its x and y extents
__device__ __forceinline__ void brick_face_box(int comp, int& oi, int& oj, int& ok, int& ex, int& ey) {
  oi = comp == 0 ? 0 : -1; oj = comp == 1 ? 0 : -1; ok = comp == 2 ? 0 : -1;
  ex = comp == 0 ? 5 : 6; ey = comp == 1 ? 5 : 6;
}
// one particle's eight terms of component comp: into the brick's faces when
// the whole stencil lies inside them, else straight to global memory
__device__ __forceinline__ void p2g_brick_comp(const Dims& d, float2* __restrict__ acc, float* sm, int comp,
                                               int fx, int fy, int fz, float x, float y, float z, float vel) {
  int i0, j0, k0; float tx, ty, tz;
  face_coords_f(d, comp, x, y, z, i0, j0, k0, tx, ty, tz);
  const float s0 = 1.f - tx, s1 = tx, t0 = 1.f - ty, t1 = ty, r0 = 1.f - tz, r1 = tz;
  const float wA = s0 * t0, wB = s1 * t0, wC = s0 * t1, wD = s1 * t1;
  const float w8[8] = { wA * r0, wB * r0, wC * r0, wD * r0, wA * r1, wB * r1, wC * r1, wD * r1 };
  int oi, oj, ok, ex, ey;
  brick_face_box(comp, oi, oj, ok, ex, ey);
  const int ez = comp == 2 ? 5 : 6;
  const int li = i0 - (fx + oi), lj = j0 - (fy + oj), lk = k0 - (fz + ok);
  if ((unsigned)li < (unsigned)(ex - 1) && (unsigned)lj < (unsigned)(ey - 1) && (unsigned)lk < (unsigned)(ez - 1)) {
    float* m = sm + comp * kBrickFaces;
    float* w = m + 3 * kBrickFaces;
    const int o = (lk * ey + lj) * ex + li, sj = ex, sk = ex * ey;
    const int o8[8] = { o, o + 1, o + sj, o + sj + 1, o + sk, o + sk + 1, o + sk + sj, o + sk + sj + 1 };
#pragma unroll
    for (int q = 0; q < 8; q++) {
      atomicAdd(&m[o8[q]], w8[q] * vel);
      atomicAdd(&w[o8[q]], w8[q]);
    }
  } else {
    long long idx, sj, sk;
    face_strides(d, comp, i0, j0, k0, idx, sj, sk);
    const long long o8[8] = { idx, idx + 1, idx + sj, idx + sj + 1, idx + sk, idx + sk + 1, idx + sk + sj,
                              idx + sk + sj + 1 };
#pragma unroll
    for (int q = 0; q < 8; q++) atomicAdd(&acc[o8[q]], make_float2(w8[q] * vel, w8[q]));
  }
}
// One block per brick (the brick list, or every brick when allBricks). The
// brick's particle range is cut into 32 lane chunks, so the 32 lanes of a
// warp work on particles about a 32nd of the range apart, mostly in
// different cells, and their shared-memory adds rarely meet on one address.
__global__ void __launch_bounds__(256) k_p2g_bricks(Dims d, GridDev g, PartsDev P, CellSort cs, BrickSet B,
                                                    int allBricks, int* err) {
  __shared__ float sm[6 * kBrickFaces];
  const int nB = allBricks ? B.nbx * B.nby * B.nbz : *B.count;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int e = blockIdx.x; e < nB; e += gridDim.x) {
    const int b = allBricks ? e : B.list[e];
    const int s0 = cs.start[b << 6], n = cs.start[(b << 6) + 64] - s0;
    if (n <= 0) continue;                              // uniform over the block
    if (threadIdx.x < 64) cs.count[(b << 6) + threadIdx.x] = 0;   // zero again for the next binning
    if (s0 < 0 || s0 + n > cs.cap) { if (threadIdx.x == 0) atomicOr(err, WS_DERR_RANGE); continue; }
    int bx, by, bz;
    brick_coords(B, b, bx, by, bz);
    const int fx = bx * 4, fy = by * 4, fz = bz * 4;
    for (int t = threadIdx.x; t < 6 * kBrickFaces; t += blockDim.x) sm[t] = 0.f;
    __syncthreads();
    const int L = (n + 31) >> 5;                       // lane chunk
    for (int a = warp; a < L; a += 8) {
      const int at = lane * L + a;
      if (at >= n) continue;
      const int p = cs.perm[s0 + at];
      const float x = P.px[p], y = P.py[p], z = P.pz[p];
      const float u = P.pvx[p], v = P.pvy[p], w = P.pvz[p];
      p2g_brick_comp(d, g.acc, sm, 0, fx, fy, fz, x, y, z, u);
      p2g_brick_comp(d, g.acc, sm, 1, fx, fy, fz, x, y, z, v);
      p2g_brick_comp(d, g.acc, sm, 2, fx, fy, fz, x, y, z, w);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < 3 * kBrickFaces; t += blockDim.x) {
      const float m = sm[t], wt = sm[t + 3 * kBrickFaces];
      if (wt == 0.f && m == 0.f) continue;            // a face no stencil reached
      const int comp = t / kBrickFaces, f = t - comp * kBrickFaces;
      int oi, oj, ok, ex, ey;
      brick_face_box(comp, oi, oj, ok, ex, ey);
      const int li = f % ex, lj = (f / ex) % ey, lk = f / (ex * ey);
      long long idx, sj, sk;
      face_strides(d, comp, fx + oi + li, fy + oj + lj, fz + ok + lk, idx, sj, sk);
      atomicAdd(&g.acc[idx], make_float2(m, wt));
    }
    __syncthreads();                                   // sm is cleared for the next brick
  }
}
size_t cell_sort_scratch_bytes(long long nKeys) {
  size_t bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, bytes, (const int*)nullptr, (int*)nullptr, (int)(nKeys + 1));
  return bytes;
}
// P2G in cell order. binned: the mark pass of this substep counted the
// particles (k_mark_fluid with the cell sort) and the brick list is current;
// otherwise the particles are counted here and every brick is visited.
// Returns the number of kernel launches made (-1 on a launch error).
int launch_p2g_sorted(const Dims& d, const GridDev& g, const PartsDev& P, const CellSort& cs, const BrickSet& B,
                      bool binned, void* scratch, size_t scratchBytes, DevStatus* st, cudaStream_t s) {
  if (P.nP <= 0) return 0;
  const long long nKeys = 64LL * B.nbx * B.nby * B.nbz;
  int launches = 0;
  if (!binned) {
    if (cudaMemsetAsync(cs.count, 0, sizeof(int) * (size_t)(nKeys + 1), s) != cudaSuccess) return -1;
    k_bin_cells<<<grid_for(P.nP, 256), 256, 0, s>>>(d, g, P, cs, &st->err);
    launches++;
  }
  // prefix sum over the keys (CUB's device scan, a CUDA toolkit library)
  if (cub::DeviceScan::ExclusiveSum(scratch, scratchBytes, cs.count, cs.start, (int)(nKeys + 1), s) != cudaSuccess)
    return -1;
  launches += 2;
  k_cell_scatter<<<grid_for(P.nP, 256), 256, 0, s>>>(P.nP, cs, &st->err);
  k_p2g_bricks<<<brick_grid(B), 256, 0, s>>>(d, g, P, cs, B, binned ? 0 : 1, &st->err);
  return launches + 2;
}

// Solid-adjacent interior face: the velocity of the solid cell beside it,
// the left one first (_applyBCSlice, js/solver.js:1153-1170): 0 for rock and
// the domain shell, the ball's velocity for a ball cell.
__device__ __forceinline__ float solid_face_velocity(const Dims& d, const GridDev& g, int comp, long long cL, long long cR) {
  if (!g.sv) return 0.f;
  const long long c = g.type[cL] == WS_SOLID ? cL : cR;
  return g.sv[comp * d.nCells + c];
}

// ------------------------------------------------------------ 4. faces pass 1
// _p2gNormalizeFace (:1109-1120) + _applyBC (:1130-1171)
// + FLIP snapshot (:2579) + the extrapolation valid mark (:1578-1611).
// Bytes: 8F read + 4F vel + 4F velO + 1F valid + 2 type reads per face.
__device__ __forceinline__ void face_normalize_bc(const Dims& d, const GridDev& g, long long f, const FaceIJK& F) {
  float2 a = g.acc[f];
  float u = a.x;
  if ((double)a.y > 1e-8) u = (float)((double)a.x / (double)a.y);
  long long cL = 0, cR = 0;
  bool solidAdj = face_cells(d, F, cL, cR);
  if (solidAdj) u = 0.f;                                   // domain boundary plane
  else if (g.type[cL] == WS_SOLID || g.type[cR] == WS_SOLID) { solidAdj = true; u = solid_face_velocity(d, g, F.comp, cL, cR); }
  g.vel[f] = u;
  g.velO[f] = u;
  g.valid[f] = ((double)a.y > 1e-8 || solidAdj) ? 1 : 0;
}
__global__ void k_faces_normalize_bc(Dims d, GridDev g) {
  long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (f >= d.F) return;
  face_normalize_bc(d, g, f, decode_face(d, f));
}
void launch_faces_normalize_bc(const Dims& d, const GridDev& g, cudaStream_t s) {
  k_faces_normalize_bc<<<grid_for(d.F, 256), 256, 0, s>>>(d, g);
}

// ------------------------------------------------------------ 5. forces
// _viscosity (:1259-1304, Jacobi: neighbours from the snapshot, which equals
// the post-BC field on entry), planet gravity (:1229-1256 with the ramp of
// :2656-2662 applied by the caller in gs) and the BC again (:2598).
__device__ __forceinline__ void face_forces(const Dims& d, const GridDev& g, long long f, const FaceIJK& F, double coef,
                                            int viscOn, double dt, double gs) {
  long long cL = 0, cR = 0;
  if (face_cells(d, F, cL, cR)) { g.vel[f] = 0.f; return; }
  int tL = g.type[cL], tR = g.type[cR];
  if (tL == WS_SOLID || tR == WS_SOLID) { g.vel[f] = solid_face_velocity(d, g, F.comp, cL, cR); return; }
  const float* __restrict__ o = g.velO;
  float u = o[f];
  if (viscOn && tL == WS_FLUID && tR == WS_FLUID) {
    int nx = d.nx, ny = d.ny, nz = d.nz;
    long long sI = 1, sJ, sK; int iLo, iHi, jLo, jHi, kLo, kHi;
    if (F.comp == 0) { sJ = nx + 1; sK = (long long)ny * (nx + 1);
      iLo = F.i - 1 >= 0; iHi = F.i + 1 <= nx; jLo = F.j - 1 >= 0; jHi = F.j + 1 < ny; kLo = F.k - 1 >= 0; kHi = F.k + 1 < nz; }
    else if (F.comp == 1) { sJ = nx; sK = (long long)(ny + 1) * nx;
      iLo = F.i - 1 >= 0; iHi = F.i + 1 < nx; jLo = F.j - 1 >= 0; jHi = F.j + 1 <= ny; kLo = F.k - 1 >= 0; kHi = F.k + 1 < nz; }
    else { sJ = nx; sK = (long long)ny * nx;
      iLo = F.i - 1 >= 0; iHi = F.i + 1 < nx; jLo = F.j - 1 >= 0; jHi = F.j + 1 < ny; kLo = F.k - 1 >= 0; kHi = F.k + 1 <= nz; }
    double c0 = o[f];
    double val = c0 * 6;
    val -= iLo ? (double)o[f - sI] : c0;
    val -= iHi ? (double)o[f + sI] : c0;
    val -= jLo ? (double)o[f - sJ] : c0;
    val -= jHi ? (double)o[f + sJ] : c0;
    val -= kLo ? (double)o[f - sK] : c0;
    val -= kHi ? (double)o[f + sK] : c0;
    u = (float)(c0 + coef * val);
  }
  if (gs > 0 && (tL == WS_FLUID || tR == WS_FLUID)) u = (float)((double)u + (double)g.gvel[f] * dt * gs);
  g.vel[f] = u;
}
__global__ void k_faces_forces(Dims d, GridDev g, double coef, int viscOn, double dt, double gs) {
  long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (f >= d.F) return;
  face_forces(d, g, f, decode_face(d, f), coef, viscOn, dt, gs);
}
void launch_faces_forces(const Dims& d, const GridDev& g, double coef, int viscOn, double dt, double gs, cudaStream_t s) {
  k_faces_forces<<<grid_for(d.F, 256), 256, 0, s>>>(d, g, coef, viscOn, dt, gs);
}

// ------------------------------------------------------------ 6. pressure setup
// _pressureSolve passes 1-2, js/solver.js:1321-1366: q = 0 off the fluid,
// diag = Nf + Na, rhs = -dx^2 div, relaxation weight pw = omega/diag
// (float32, as the reference's pW). pw < 0 marks a non-fluid cell. Each
// 256-cell block also counts its interior fluid cells per colour for the SOR
// list build (sorCounts[2 b], [2 b + 1]; null skips) and adds its fluid
// cells to the fluid count with one atomic.
// one cell of the setup: returns whether it is fluid and its SOR colour (-1 off the lists)
__device__ __forceinline__ bool cell_pressure_setup(const Dims& d, const GridDev& g, uint8_t* __restrict__ diag8,
                                                    double omega, long long c, int i, int j, int k, int& col) {
  col = -1;
  const uint8_t* type = g.type;
  if (type[c] != WS_FLUID) { g.q[c] = 0.f; g.pw[c] = -1.f; diag8[c] = 0; return false; }
  int nx = d.nx, ny = d.ny, nz = d.nz; long long nxy = (long long)nx * ny;
  long long nbr[6] = { i > 0 ? c - 1 : -1, i < nx - 1 ? c + 1 : -1, j > 0 ? c - nx : -1,
                       j < ny - 1 ? c + nx : -1, k > 0 ? c - nxy : -1, k < nz - 1 ? c + nxy : -1 };
  int cnt = 0;
#pragma unroll
  for (int q = 0; q < 6; q++) if (nbr[q] >= 0 && type[nbr[q]] != WS_SOLID) cnt++;
  const float* u = g.vel; const float* v = g.vel + d.uN; const float* w = g.vel + d.uN + d.vN;
  double div = ((double)u[((long long)k * ny + j) * (nx + 1) + i + 1] - (double)u[((long long)k * ny + j) * (nx + 1) + i] +
                (double)v[((long long)k * (ny + 1) + j + 1) * nx + i] - (double)v[((long long)k * (ny + 1) + j) * nx + i] +
                (double)w[((long long)(k + 1) * ny + j) * nx + i] - (double)w[((long long)k * ny + j) * nx + i]) / d.dx;
  g.rhs[c] = (float)(-d.dx * d.dx * div);
  g.pw[c] = (float)(cnt > 0 ? omega / (double)cnt : 0.0);
  diag8[c] = (uint8_t)cnt;
  // membership of the SOR colour lists: interior fluid cells (sor_colour)
  if (i >= 1 && j >= 1 && k >= 1 && i + 2 <= nx && j + 2 <= ny && k + 2 <= nz) col = (i + j + k) & 1;
  return true;
}
__global__ void __launch_bounds__(256) k_pressure_setup(Dims d, GridDev g, uint8_t* __restrict__ diag8, double omega,
                                                        DevStatus* st, int* __restrict__ sorCounts) {
  __shared__ int wc[3][8];                           // per warp: colour-0 and colour-1 list cells, fluid cells
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  int col = -1, fluid = 0;
  if (c < d.nCells) {
    int i, j, k; decode_cell(d, c, i, j, k);
    fluid = cell_pressure_setup(d, g, diag8, omega, c, i, j, k, col) ? 1 : 0;
  }
  const unsigned full = 0xffffffffu;
  const unsigned m0 = __ballot_sync(full, col == 0), m1 = __ballot_sync(full, col == 1), mf = __ballot_sync(full, fluid);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { wc[0][wid] = __popc(m0); wc[1][wid] = __popc(m1); wc[2][wid] = __popc(mf); }
  __syncthreads();
  if (threadIdx.x == 0) {
    int a = 0, b = 0, f = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) { a += wc[0][q]; b += wc[1][q]; f += wc[2][q]; }
    if (sorCounts) { sorCounts[2 * blockIdx.x] = a; sorCounts[2 * blockIdx.x + 1] = b; }
    if (f) atomicAdd(&st->nFluid, f);
  }
}
void launch_pressure_setup(const Dims& d, const GridDev& g, uint8_t* diag8, double omega, DevStatus* st, int* sorCounts,
                           cudaStream_t s) {
  k_pressure_setup<<<grid_for(d.nCells, 256), 256, 0, s>>>(d, g, diag8, omega, st, sorCounts);
}

// ------------------------------------------------------------ 7. red-black SOR
// One colour of the SOR sweep, js/solver.js:1397-1404 in red-black order:
// q <- q (1 - omega) + pw (rhs + sum of the six neighbour q), FP64 arithmetic
// rounded to float32 as the reference's Float32Array store. q is zero on
// every non-fluid cell, so summing all six neighbours in the reference's
// order (-x, +x, -y, +y, -z, +z) equals its sum over fluid neighbours.
// The thread layout packs the cells of one colour: thread t -> row r, slot s,
// i = 2 s + ((j + k + colour) & 1). Bytes per full iteration: 13 per cell.
__global__ void k_sor_color(Dims d, float* __restrict__ q, const float* __restrict__ rhs,
                            const float* __restrict__ pw, int color, double om1) {
  int nx = d.nx, ny = d.ny, nz = d.nz;
  int half = (nx + 1) >> 1;
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long rows = (long long)ny * nz;
  if (t >= rows * half) return;
  int sl = (int)(t % half); long long r = t / half;
  int j = (int)(r % ny), k = (int)(r / ny);
  int i = 2 * sl + ((j + k + color) & 1);
  if (i >= nx) return;
  long long c = r * nx + i;
  float w = pw[c];
  if (w < 0.f) return;
  if (i < 1 || i > nx - 2 || j < 1 || j > ny - 2 || k < 1 || k > nz - 2) return;
  long long nxy = (long long)nx * ny;
  q[c] = sor_update(q[c], w, rhs[c], q[c - 1], q[c + 1], q[c - nx], q[c + nx], q[c - nxy], q[c + nxy], om1);
}
void launch_sor_color(const Dims& d, const GridDev& g, int color, double om1, cudaStream_t s) {
  long long n = (long long)d.ny * d.nz * ((d.nx + 1) >> 1);
  k_sor_color<<<grid_for(n, 256), 256, 0, s>>>(d, g.q, g.rhs, g.pw, color, om1);
}

// ------------------------------------------------------------ 8. FP64 residual
// ||b - A q||_2 / ||b||_2 over fluid cells with A, b the reference assembly
// (js/solver.js:1361-1365): r = rhs + sum_fluid q_n - diag q. Block partials
// in FP64, combined in a fixed order by k_residual_final (deterministic).
__global__ void k_residual_partial(Dims d, const float* __restrict__ q, const float* __restrict__ rhs,
                                   const float* __restrict__ pw, const uint8_t* __restrict__ diag8,
                                   double2* __restrict__ partials) {
  __shared__ double srr[32], sbb[32];
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double rr = 0, bb = 0;
  bool interior = false;
  if (c < d.nCells) {
    int i, j, k; decode_cell(d, c, i, j, k);
    interior = i > 0 && i < d.nx - 1 && j > 0 && j < d.ny - 1 && k > 0 && k < d.nz - 1;
  }
  if (interior && pw[c] >= 0.f) {
    int nx = d.nx; long long nxy = (long long)nx * d.ny;
    double sum = (double)q[c - 1];
    sum += (double)q[c + 1]; sum += (double)q[c - nx]; sum += (double)q[c + nx];
    sum += (double)q[c - nxy]; sum += (double)q[c + nxy];
    double b = rhs[c];
    double r = b + sum - (double)diag8[c] * (double)q[c];
    rr = r * r; bb = b * b;
  }
  rr = warp_sum(rr); bb = warp_sum(bb);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { srr[wid] = rr; sbb[wid] = bb; }
  __syncthreads();
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    rr = lane < nw ? srr[lane] : 0; bb = lane < nw ? sbb[lane] : 0;
    rr = warp_sum(rr); bb = warp_sum(bb);
    if (lane == 0) partials[blockIdx.x] = make_double2(rr, bb);
  }
}
__global__ void k_residual_final(const double2* __restrict__ partials, int n, DevStatus* st, double* hostMirror) {
  __shared__ double srr[32], sbb[32];
  double rr = 0, bb = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) { rr += partials[i].x; bb += partials[i].y; }
  rr = warp_sum(rr); bb = warp_sum(bb);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { srr[wid] = rr; sbb[wid] = bb; }
  __syncthreads();
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    rr = lane < nw ? srr[lane] : 0; bb = lane < nw ? sbb[lane] : 0;
    rr = warp_sum(rr); bb = warp_sum(bb);
    if (lane == 0) {
      double rel = bb > 0 ? sqrt(rr) / sqrt(bb) : sqrt(rr);
      st->rr = rr; st->bb = bb; st->relres = rel;
      if (hostMirror) *hostMirror = rel;
    }
  }
}
int residual_blocks(const Dims& d) { return (int)grid_for(d.nCells, 256); }
void launch_residual(const Dims& d, const GridDev& g, const uint8_t* diag8, double2* partials,
                     DevStatus* st, double* hostMirror, cudaStream_t s) {
  int nb = residual_blocks(d);
  k_residual_partial<<<nb, 256, 0, s>>>(d, g.q, g.rhs, g.pw, diag8, partials);
  k_residual_final<<<1, 1024, 0, s>>>(partials, nb, st, hostMirror);
}

// ------------------------------------------------------------ 9. project (+clamp)
// _projectSlice (:1417-1443) and, fused when vorticity is off,
// _clampUmSlice (:2629-2653) with the max |u| reduction (exact: max of
// non-negative float bit patterns).
// block-level max, then one atomic per block (every thread of the block must call)
__device__ __forceinline__ void umax_reduce(float a, DevStatus* st) {
  __shared__ unsigned sm[32];
  unsigned bits = __float_as_uint(fabsf(a));
  bits = warp_max_u(bits);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sm[wid] = bits;
  __syncthreads();
  if (wid == 0) {
    bits = lane < (int)(blockDim.x >> 5) ? sm[lane] : 0u;
    bits = warp_max_u(bits);
    if (lane == 0 && bits) atomicMax(&st->umaxBits, bits);
  }
}
__device__ __forceinline__ float face_project(const Dims& d, const GridDev& g, long long f, const FaceIJK& F, int doClamp,
                                              float vcap) {
  float u = g.vel[f];
  long long cL = 0, cR = 0;
  if (!face_cells(d, F, cL, cR)) {
    int tL = g.type[cL], tR = g.type[cR];
    if (tL != WS_SOLID && tR != WS_SOLID) {
      double pL = tL == WS_FLUID ? (double)g.q[cL] : 0.0, pR = tR == WS_FLUID ? (double)g.q[cR] : 0.0;
      u = (float)((double)u - (pR - pL) * (1.0 / d.dx));
    }
  }
  if (doClamp) { if (u > vcap) u = vcap; else if (u < -vcap) u = -vcap; }
  g.vel[f] = u;
  return u;
}
__global__ void k_project(Dims d, GridDev g, int doClamp, float vcap, DevStatus* st) {
  long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  float u = 0.f;
  if (f < d.F) u = face_project(d, g, f, decode_face(d, f), doClamp, vcap);
  if (doClamp) umax_reduce(u, st);
}
void launch_project(const Dims& d, const GridDev& g, int doClamp, double maxSpeed, DevStatus* st, cudaStream_t s) {
  k_project<<<grid_for(d.F, 256), 256, 0, s>>>(d, g, doClamp, (float)(maxSpeed * 1.1), st);
}
__global__ void k_clamp_umax(Dims d, float* __restrict__ vel, float vcap, DevStatus* st) {
  long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  float u = 0.f;
  if (f < d.F) {
    u = vel[f];
    if (u > vcap) { u = vcap; vel[f] = u; } else if (u < -vcap) { u = -vcap; vel[f] = u; }
  }
  umax_reduce(u, st);
}
void launch_clamp_umax(const Dims& d, const GridDev& g, double maxSpeed, DevStatus* st, cudaStream_t s) {
  k_clamp_umax<<<grid_for(d.F, 256), 256, 0, s>>>(d, g.vel, (float)(maxSpeed * 1.1), st);
}

// ------------------------------------------------------------ 10. vorticity
// _vorticityConfinement, js/solver.js:1454-1559. (a) omega per cell from the
// float32 cell-centred velocities (recomputed from the faces, rounded as the
// reference stores them), (b) the gated confinement force per fluid cell,
// (c) the splat onto faces between two fluid cells.
// cell-centred velocities of cell (i, j, k), as the reference's _vcx/_vcy/_vcz
// (float stores of the two-face means)
__device__ __forceinline__ float ccx(const Dims& d, const float* u, int i, int j, int k) {
  const long long ui = ((long long)k * d.ny + j) * (d.nx + 1) + i;
  return (float)(0.5 * ((double)u[ui] + (double)u[ui + 1]));
}
__device__ __forceinline__ float ccy(const Dims& d, const float* v, int i, int j, int k) {
  const long long vi = ((long long)k * (d.ny + 1) + j) * d.nx + i;
  return (float)(0.5 * ((double)v[vi] + (double)v[vi + d.nx]));
}
__device__ __forceinline__ float ccz(const Dims& d, const float* w, int i, int j, int k) {
  const long long c = ((long long)k * d.ny + j) * d.nx + i, nxy = (long long)d.nx * d.ny;
  return (float)(0.5 * ((double)w[c] + (double)w[c + nxy]));
}
// Omega is read only at fluid cells: k_vort_force reads omg and om* at a fluid
// cell, and omg at its six neighbours only when all six are fluid.
__global__ void k_vort_omega(Dims d, GridDev g) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= d.nCells || g.type[c] != WS_FLUID) return;
  int nx = d.nx, ny = d.ny, nz = d.nz;
  int i, j, k; decode_cell(d, c, i, j, k);
  const float* u = g.vel; const float* v = g.vel + d.uN; const float* w = g.vel + d.uN + d.vN;
  // the clamped neighbours of the reference's central differences (a boundary cell uses itself)
  const int im = i > 0 ? i - 1 : i, ip = i < nx - 1 ? i + 1 : i;
  const int jm = j > 0 ? j - 1 : j, jp = j < ny - 1 ? j + 1 : j;
  const int km = k > 0 ? k - 1 : k, kp = k < nz - 1 ? k + 1 : k;
  double inv2 = 0.5 / d.dx;
  double wx = ((double)ccz(d, w, i, jp, k) - (double)ccz(d, w, i, jm, k) -
               ((double)ccy(d, v, i, j, kp) - (double)ccy(d, v, i, j, km))) * inv2;
  double wy = ((double)ccx(d, u, i, j, kp) - (double)ccx(d, u, i, j, km) -
               ((double)ccz(d, w, ip, j, k) - (double)ccz(d, w, im, j, k))) * inv2;
  double wz = ((double)ccy(d, v, ip, j, k) - (double)ccy(d, v, im, j, k) -
               ((double)ccx(d, u, i, jp, k) - (double)ccx(d, u, i, jm, k))) * inv2;
  g.omx[c] = (float)wx; g.omy[c] = (float)wy; g.omz[c] = (float)wz;
  g.omg[c] = (float)sqrt(wx * wx + wy * wy + wz * wz);
}
__global__ void k_vort_force(Dims d, GridDev g, double eps, double dt) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= d.nCells) return;
  const uint8_t* type = g.type;
  if (type[c] != WS_FLUID) return;
  int nx = d.nx, ny = d.ny, nz = d.nz; long long nxy = (long long)nx * ny;
  int i, j, k; decode_cell(d, c, i, j, k);
  const float* omg = g.omg;
  if (omg[c] < 0.35f ||
      (i > 0 && type[c - 1] != WS_FLUID) || (i < nx - 1 && type[c + 1] != WS_FLUID) ||
      (j > 0 && type[c - nx] != WS_FLUID) || (j < ny - 1 && type[c + nx] != WS_FLUID) ||
      (k > 0 && type[c - nxy] != WS_FLUID) || (k < nz - 1 && type[c + nxy] != WS_FLUID)) {
    g.vfx[c] = 0.f; g.vfy[c] = 0.f; g.vfz[c] = 0.f; return;
  }
  double gx = (double)omg[i < nx - 1 ? c + 1 : c] - (double)omg[i > 0 ? c - 1 : c];
  double gy = (double)omg[j < ny - 1 ? c + nx : c] - (double)omg[j > 0 ? c - nx : c];
  double gz = (double)omg[k < nz - 1 ? c + nxy : c] - (double)omg[k > 0 ? c - nxy : c];
  double g2 = gx * gx + gy * gy + gz * gz;
  if (g2 < 1e-12) { g.vfx[c] = 0.f; g.vfy[c] = 0.f; g.vfz[c] = 0.f; return; }
  double inv = 1 / sqrt(g2);
  double Nx = gx * inv, Ny = gy * inv, Nz = gz * inv;
  double ox = g.omx[c], oy = g.omy[c], oz = g.omz[c];
  double fx = eps * (Ny * oz - Nz * oy), fy = eps * (Nz * ox - Nx * oz), fz = eps * (Nx * oy - Ny * ox);
  double f2 = fx * fx + fy * fy + fz * fz, fCap = 6.0;
  if (f2 > fCap * fCap) { double fs = fCap / sqrt(f2); fx *= fs; fy *= fs; fz *= fs; }
  g.vfx[c] = (float)(fx * dt); g.vfy[c] = (float)(fy * dt); g.vfz[c] = (float)(fz * dt);
}
__global__ void k_vort_splat(Dims d, GridDev g) {
  long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (f >= d.F) return;
  FaceIJK F = decode_face(d, f);
  long long cL = 0, cR = 0;
  if (face_cells(d, F, cL, cR)) return;
  if (g.type[cL] != WS_FLUID || g.type[cR] != WS_FLUID) return;
  const float* fv = F.comp == 0 ? g.vfx : (F.comp == 1 ? g.vfy : g.vfz);
  g.vel[f] = (float)((double)g.vel[f] + 0.5 * ((double)fv[cL] + (double)fv[cR]));
}
void launch_vorticity(const Dims& d, const GridDev& g, double eps, double dt, cudaStream_t s) {
  k_vort_omega<<<grid_for(d.nCells, 256), 256, 0, s>>>(d, g);
  k_vort_force<<<grid_for(d.nCells, 256), 256, 0, s>>>(d, g, eps, dt);
  k_vort_splat<<<grid_for(d.F, 256), 256, 0, s>>>(d, g);
}

// ------------------------------------------------------------ 11. extrapolate
// _extrapolate, js/solver.js:1562-1636 in Jacobi order: an invalid face takes
// the mean of the neighbours (same component grid) that were valid before
// the pass, summed in the reference's order -i, +i, -j, +j, -k, +k. Filled
// faces are marked 2 so no thread reads a value written in this pass.
__device__ __forceinline__ void face_extrapolate(const Dims& d, const GridDev& g, long long f, const FaceIJK& F) {
  const uint8_t* valid = g.valid;
  int d0, d1, d2;
  if (F.comp == 0) { d0 = d.nx + 1; d1 = d.ny; d2 = d.nz; }
  else if (F.comp == 1) { d0 = d.nx; d1 = d.ny + 1; d2 = d.nz; }
  else { d0 = d.nx; d1 = d.ny; d2 = d.nz + 1; }
  long long sK = (long long)d0 * d1;
  const float* a = g.vel;
  // every in-range neighbour's flag and velocity in one round trip, then the
  // sum over the originally valid ones in the fixed order -x, +x, -y, +y, -z, +z
  const long long o[6] = { f - 1, f + 1, f - d0, f + d0, f - sK, f + sK };
  const bool in[6] = { F.i > 0, F.i < d0 - 1, F.j > 0, F.j < d1 - 1, F.k > 0, F.k < d2 - 1 };
  uint8_t vv[6]; float av[6];
#pragma unroll
  for (int q = 0; q < 6; q++) { vv[q] = in[q] ? valid[o[q]] : (uint8_t)0; av[q] = in[q] ? a[o[q]] : 0.f; }
  double sum = 0; int cnt = 0;
#pragma unroll
  for (int q = 0; q < 6; q++) if (vv[q] == 1) { sum += av[q]; cnt++; }
  if (cnt > 0) { g.vel[f] = (float)(sum / cnt); g.valid[f] = 2; }
}
__global__ void k_extrapolate(Dims d, GridDev g) {
  long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (f >= d.F) return;
  if (g.valid[f] != 0) return;
  face_extrapolate(d, g, f, decode_face(d, f));
}
void launch_extrapolate(const Dims& d, const GridDev& g, cudaStream_t s) {
  k_extrapolate<<<grid_for(d.F, 256), 256, 0, s>>>(d, g);
}

// ------------------------------------------------------------ active bricks
// Faces and cells far from every particle and moving solid hold fixed values
// (zero velocity, the static valid flags, q = 0 and pw = -1 off the fluid), so
// a full pass over them rewrites what is already there. The substep therefore
// runs its face and cell passes over a list of 4^3 bricks: those within one
// brick of a particle's or moving solid's cell this substep (the reach of
// P2G's stencils, the extrapolation layer and G2P's midpoint sample is under
// four cells), plus those active in the previous substep, so a brick that
// empties is rewritten once to the fixed values. A forced full pass (after a
// caller wrote grid fields) processes every brick.
__global__ void k_brick_activity(int nbx, int nby, int nbz, const uint8_t* __restrict__ seed, uint8_t* __restrict__ act,
                                 uint8_t* __restrict__ proc, const int* __restrict__ forceAll, int* __restrict__ list,
                                 int* __restrict__ count) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  const int nB = nbx * nby * nbz;
  int p = 0;
  if (b < nB) {
    const int bx = b % nbx, t = b / nbx, by = t % nby, bz = t / nby;
    int a = 0;
    for (int dz = -1; dz <= 1 && !a; dz++) {
      const int z = bz + dz;
      if (z < 0 || z >= nbz) continue;
      for (int dy = -1; dy <= 1 && !a; dy++) {
        const int y = by + dy;
        if (y < 0 || y >= nby) continue;
        const uint8_t* row = seed + ((long long)z * nby + y) * nbx;
        for (int dx = -1; dx <= 1; dx++) {
          const int x = bx + dx;
          if (x >= 0 && x < nbx && row[x]) { a = 1; break; }
        }
      }
    }
    p = a | act[b] | (*forceAll != 0);
    proc[b] = (uint8_t)p;
    act[b] = (uint8_t)a;
  }
  // the work list: one atomic per warp (the passes over it do not depend on its order)
  const unsigned m = __ballot_sync(0xffffffffu, p != 0);
  const int lane = threadIdx.x & 31;
  int base = 0;
  if (lane == 0 && m) base = atomicAdd(count, __popc(m));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (p) list[base + __popc(m & ((1u << lane) - 1u))] = b;
}
// the count reset, activity and work list, then the seeds and the
// forced-pass flag cleared for the next substep
cudaError_t launch_brick_activity(const BrickSet& B, cudaStream_t s) {
  const int nB = B.nbx * B.nby * B.nbz;
  cudaError_t e = cudaMemsetAsync(B.count, 0, sizeof(int), s);
  if (e != cudaSuccess) return e;
  k_brick_activity<<<grid_for(nB, 256), 256, 0, s>>>(B.nbx, B.nby, B.nbz, B.seed, B.act, B.proc, B.forceAll, B.list,
                                                      B.count);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(B.seed, 0, (size_t)nB, s)) != cudaSuccess) return e;
  return cudaMemsetAsync(B.forceAll, 0, sizeof(int), s);
}

// The faces a brick owns: per component, the 64 faces whose lower cell lies
// in the brick, and on the last brick along the component's axis the 16
// faces of the domain's upper plane. Slot t in [0, 240): its component and
// offsets in the brick are the same for every brick, so a thread decodes
// them once (face_slot) and each brick adds only its coordinates.
struct FaceSlot { int comp, la, lb, lc; bool upper; };
__device__ __forceinline__ FaceSlot face_slot(int t) {
  FaceSlot sl;
  sl.comp = t >= 160 ? 2 : t >= 80 ? 1 : 0;
  const int s = t - sl.comp * 80;
  sl.upper = s >= 64;
  if (!sl.upper) { sl.la = s & 3; sl.lb = (s >> 2) & 3; sl.lc = s >> 4; }
  else { sl.la = 0; sl.lb = (s - 64) & 3; sl.lc = (s - 64) >> 2; }
  return sl;
}
__device__ __forceinline__ bool brick_face(const Dims& d, const BrickSet& B, int bx, int by, int bz, const FaceSlot& sl,
                                           long long& f, FaceIJK& F) {
  const int comp = sl.comp, la = sl.la, lb = sl.lb, lc = sl.lc;
  const bool upper = sl.upper;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  F.comp = comp;
  if (comp == 0) {
    if (upper && bx != B.nbx - 1) return false;
    F.i = upper ? nx : bx * 4 + la; F.j = by * 4 + lb; F.k = bz * 4 + lc;
    if ((!upper && F.i >= nx) || F.j >= ny || F.k >= nz) return false;
    f = ((long long)F.k * ny + F.j) * (nx + 1) + F.i;
  } else if (comp == 1) {
    if (upper && by != B.nby - 1) return false;
    F.j = upper ? ny : by * 4 + la; F.i = bx * 4 + lb; F.k = bz * 4 + lc;
    if ((!upper && F.j >= ny) || F.i >= nx || F.k >= nz) return false;
    f = d.uN + ((long long)F.k * (ny + 1) + F.j) * nx + F.i;
  } else {
    if (upper && bz != B.nbz - 1) return false;
    F.k = upper ? nz : bz * 4 + la; F.i = bx * 4 + lb; F.j = by * 4 + lc;
    if ((!upper && F.k >= nz) || F.i >= nx || F.j >= ny) return false;
    f = d.uN + d.vN + ((long long)F.k * ny + F.j) * nx + F.i;
  }
  F.local = 0;
  return true;
}

// one face pass over the brick list (persistent blocks, one brick per
// iteration); op 0 normalise + BC, 1 forces, 2 project (+ clamp, umax),
// 3 extrapolate, 4 clear the P2G accumulator
struct FacePassArgs { double coef, dt, gs; int viscOn, doClamp; float vcap; };
template <int OP>
__global__ void __launch_bounds__(256) k_faces_bricks(Dims d, GridDev g, BrickSet B, FacePassArgs fa, DevStatus* st) {
  if (OP == 4 && *B.forceAll) {                          // after a forced full pass: the whole accumulator
    const long long F2 = d.F >> 1;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t <= F2; t += (long long)gridDim.x * blockDim.x) {
      if (t < F2) reinterpret_cast<float4*>(g.acc)[t] = make_float4(0.f, 0.f, 0.f, 0.f);
      else if (d.F & 1) g.acc[d.F - 1] = make_float2(0.f, 0.f);
    }
    return;
  }
  const int n = *B.count;
  float umax = 0.f;
  const FaceSlot sl = face_slot(threadIdx.x < 240 ? (int)threadIdx.x : 0);
  int b = (int)blockIdx.x < n ? B.list[blockIdx.x] : 0;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    // the next brick's id is loaded before this brick's faces are touched, so
    // its round trip overlaps this brick's loads and stores
    const int bNext = it + (int)gridDim.x < n ? B.list[it + gridDim.x] : 0;
    long long f; FaceIJK F;
    int bx, by, bz;
    brick_coords(B, b, bx, by, bz);
    if (threadIdx.x < 240 && brick_face(d, B, bx, by, bz, sl, f, F)) {
      if (OP == 0) face_normalize_bc(d, g, f, F);
      else if (OP == 1) face_forces(d, g, f, F, fa.coef, fa.viscOn, fa.dt, fa.gs);
      else if (OP == 2) umax = fmaxf(umax, fabsf(face_project(d, g, f, F, fa.doClamp, fa.vcap)));
      else if (OP == 3) { if (g.valid[f] == 0) face_extrapolate(d, g, f, F); }
      else g.acc[f] = make_float2(0.f, 0.f);
    }
    b = bNext;
  }
  if (OP == 2 && fa.doClamp) umax_reduce(umax, st);
}
static unsigned brick_grid(const BrickSet& B) {
  const int nB = B.nbx * B.nby * B.nbz;
  return (unsigned)std::min(nB, 148 * 8);
}
void launch_faces_normalize_bc_bricks(const Dims& d, const GridDev& g, const BrickSet& B, cudaStream_t s) {
  k_faces_bricks<0><<<brick_grid(B), 256, 0, s>>>(d, g, B, FacePassArgs{}, nullptr);
}
void launch_faces_forces_bricks(const Dims& d, const GridDev& g, const BrickSet& B, double coef, int viscOn, double dt,
                                double gs, cudaStream_t s) {
  FacePassArgs fa{}; fa.coef = coef; fa.viscOn = viscOn; fa.dt = dt; fa.gs = gs;
  k_faces_bricks<1><<<brick_grid(B), 256, 0, s>>>(d, g, B, fa, nullptr);
}
void launch_project_bricks(const Dims& d, const GridDev& g, const BrickSet& B, int doClamp, double maxSpeed,
                           DevStatus* st, cudaStream_t s) {
  FacePassArgs fa{}; fa.doClamp = doClamp; fa.vcap = (float)(maxSpeed * 1.1);
  k_faces_bricks<2><<<brick_grid(B), 256, 0, s>>>(d, g, B, fa, st);
}
void launch_extrapolate_bricks(const Dims& d, const GridDev& g, const BrickSet& B, cudaStream_t s) {
  k_faces_bricks<3><<<brick_grid(B), 256, 0, s>>>(d, g, B, FacePassArgs{}, nullptr);
}
// the accumulator of the bricks in the list (those the previous substep's
// P2G may have written), or all of it after a forced full pass
void launch_clear_acc_bricks(const Dims& d, const GridDev& g, const BrickSet& B, cudaStream_t s) {
  k_faces_bricks<4><<<brick_grid(B), 256, 0, s>>>(d, g, B, FacePassArgs{}, nullptr);
}
// the pressure setup over the brick list: four bricks per 256-thread block
__global__ void __launch_bounds__(256) k_pressure_setup_bricks(Dims d, GridDev g, uint8_t* __restrict__ diag8,
                                                               double omega, DevStatus* st, BrickSet B) {
  const int n = *B.count;
  int fluid = 0;
  for (int it = blockIdx.x * 4; it < n; it += gridDim.x * 4) {
    const int e = it + (threadIdx.x >> 6);
    if (e >= n) continue;
    const int b = B.list[e], c = threadIdx.x & 63;
    int bx, by, bz;
    brick_coords(B, b, bx, by, bz);
    const int i = bx * 4 + (c & 3), j = by * 4 + ((c >> 2) & 3), k = bz * 4 + (c >> 4);
    if (i >= d.nx || j >= d.ny || k >= d.nz) continue;
    int col;
    if (cell_pressure_setup(d, g, diag8, omega, ((long long)k * d.ny + j) * d.nx + i, i, j, k, col)) fluid++;
  }
  fluid = warp_sum(fluid);
  if ((threadIdx.x & 31) == 0 && fluid) atomicAdd(&st->nFluid, fluid);
}
void launch_pressure_setup_bricks(const Dims& d, const GridDev& g, uint8_t* diag8, double omega, DevStatus* st,
                                  const BrickSet& B, cudaStream_t s) {
  k_pressure_setup_bricks<<<brick_grid(B), 256, 0, s>>>(d, g, diag8, omega, st, B);
}

// ------------------------------------------------------------ field helpers
__global__ void k_extract_weight(Dims d, const float2* __restrict__ acc, float* __restrict__ out, long long off, long long n) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < n) out[t] = acc[off + t].y;
}
void launch_extract_weight(const Dims& d, const float2* acc, float* out, long long off, long long n, cudaStream_t s) {
  k_extract_weight<<<grid_for(n, 256), 256, 0, s>>>(d, acc, out, off, n);
}
