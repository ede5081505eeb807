// ws_queries.cu — the FluidSolver helpers callers poll or fire between
// steps: waveImpulse (js/solver.js:3866-3892), dryLandFraction (:3593-3623),
// sampleVel (:811-854), terrainRadiusAt (:512-535) and oceanPoint (:591-608).
//
// waveImpulse and oceanPoint draw from Math.random() in the reference, an
// unseeded generator. Here they draw from the handle's seeded stir stream
// (stirS, the same LCG and [0, 1) mapping as the reference's seeded
// streams), so a call is reproducible and the oracle restates it draw for
// draw. waveImpulse: two draws pick the bulge direction, then particle p
// takes draw p + 1 of the stream that follows (whether or not it is
// pushed), so every particle's draw is known without a scan; the stream
// then stands nP draws further on. oceanPoint: attempt a takes draws 2a + 1
// and 2a + 2, and the stream advances by two draws per attempt made.
#include "ws_kernels.cuh"

// waveImpulse, sphere mode: a radial push on the bulge side, strongest where
// the surface faces the bulge direction (dir), random factor 0.7..1.0
__global__ void k_wave_impulse(Dims d, PartsDev P, double dirx, double diry, double dirz, uint32_t s0, double dvx) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nP) return;
  const double ex = (double)P.px[p] - d.cx, ey = (double)P.py[p] - d.cy, ez = (double)P.pz[p] - d.cz;
  double er = sqrt(ex * ex + ey * ey + ez * ez);
  if (er == 0 || isnan(er)) er = 1e-9;                  // `|| 1e-9`
  const double pr = (ex * dirx + ey * diry + ez * dirz) / er;
  if (pr <= 0) return;
  const double rnd = lcg_jump(s0, (uint32_t)p + 1u) / 4294967296.0;
  const double f = pr * pr * pr * (0.7 + rnd * 0.3);
  P.pvx[p] = (float)((double)P.pvx[p] + ex / er * dvx * f);
  P.pvy[p] = (float)((double)P.pvy[p] + ey / er * dvx * f);
  P.pvz[p] = (float)((double)P.pvz[p] + ez / er * dvx * f);
}
void launch_wave_impulse(const Dims& d, const PartsDev& P, const double dir[3], uint32_t s0, double dvx, cudaStream_t s) {
  if (P.nP <= 0) return;
  k_wave_impulse<<<grid_for(P.nP, 256), 256, 0, s>>>(d, P, dir[0], dir[1], dir[2], s0, dvx);
}

// dryLandFraction: 1200 golden-angle rays, one thread each; a ray is dry when
// its rock surface stands above sea level and the first open cell above it
// holds no fluid. Exact integer count.
__global__ void k_dry_land(Dims d, TerrainDev t, const uint8_t* __restrict__ type, double oceanR, int* dry) {
  const int N = 1200;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int isDry = 0;
  if (i < N) {
    const double a = i * 2.399963, u = 1 - 2 * (i + 0.5) / N;
    const double sq = sqrt(1 - u * u);
    const double ldx = sq * cos(a), ldy = u, ldz = sq * sin(a);
    const int n = t.n;
    double Rt = -1;
    for (double rr = t.Rhi + t.dv; rr > t.Rlo - t.dv; rr -= t.dv * 0.5) {
      const int sx = jtrunc(over_dv(t, d.cx + ldx * rr)), sy = jtrunc(over_dv(t, d.cy + ldy * rr)),
                sz = jtrunc(over_dv(t, d.cz + ldz * rr));
      if (sx < 0 || sy < 0 || sz < 0 || sx >= n || sy >= n || sz >= n) continue;
      if (t.solid[((long long)sz * n + sy) * n + sx]) { Rt = rr; break; }
    }
    if (!(Rt < 0 || Rt <= oceanR)) {
      bool wet = false;
      for (int st = 1; st <= 4; st++) {
        const double rp = Rt + st * d.dx * 0.55;
        const int ii = jtrunc(over_dx(d, d.cx + ldx * rp)), jj = jtrunc(over_dx(d, d.cy + ldy * rp)),
                  kk = jtrunc(over_dx(d, d.cz + ldz * rp));
        if (ii < 0 || jj < 0 || kk < 0 || ii >= d.nx || jj >= d.ny || kk >= d.nz) break;
        const int ct = type[((long long)kk * d.ny + jj) * d.nx + ii];
        if (ct == WS_SOLID) continue;
        if (ct == WS_FLUID) wet = true;
        break;                                           // the first open cell decides
      }
      isDry = wet ? 0 : 1;
    }
  }
  isDry = warp_sum(isDry);
  if ((threadIdx.x & 31) == 0 && isDry) atomicAdd(dry, isDry);
}
void launch_dry_land(const Dims& d, const TerrainDev& t, const uint8_t* type, double oceanR, int* dry, cudaStream_t s) {
  cudaMemsetAsync(dry, 0, sizeof(int), s);
  k_dry_land<<<grid_for(1200, 128), 128, 0, s>>>(d, t, type, oceanR, dry);
}

// sampleVel at n points (x, y, z triples): the trilinear MAC sample of the
// current face velocities, in double
__global__ void k_sample_vel(Dims d, const float* __restrict__ vel, const double* __restrict__ xyz, long long n,
                             double* __restrict__ out) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double a, b, c;
  sample_vel3(d, vel, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], a, b, c);
  out[3 * i] = a; out[3 * i + 1] = b; out[3 * i + 2] = c;
}
void launch_sample_vel(const Dims& d, const float* vel, const double* xyz, long long n, double* out, cudaStream_t s) {
  if (n <= 0) return;
  k_sample_vel<<<grid_for(n, 256), 256, 0, s>>>(d, vel, xyz, n, out);
}

// terrainRadiusAt at n points: the trilinear terrain radius (coreR without terrain)
__global__ void k_terrain_radius(TerrainDev t, double coreR, const double* __restrict__ xyz, long long n,
                                 double* __restrict__ out) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = terrain_radius_at(t, coreR, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
}
void launch_terrain_radius(const TerrainDev& t, double coreR, const double* xyz, long long n, double* out,
                           cudaStream_t s) {
  if (n <= 0) return;
  k_terrain_radius<<<grid_for(n, 256), 256, 0, s>>>(t, coreR, xyz, n, out);
}

// oceanPoint: the 64 attempts in parallel (one lane each), then the
// reference's choice: the first attempt deeper than `need` returns at once,
// else the deepest (first of equals) when deeper than -1, else the point above
// the centre at sea level. out: x, y, z and the number of attempts made.
__global__ void k_ocean_point(Dims d, TerrainDev t, double coreR, double oceanR, double need, uint32_t s0,
                              double* out) {
  __shared__ double dpt[64], px[64], py[64], pz[64];
  const int a = threadIdx.x;
  {
    const uint32_t s1 = lcg_jump(s0, 2u * a + 1u), s2 = lcg_next(s1);
    const double u1 = s1 / 4294967296.0 * 2 - 1, th = s2 / 4294967296.0 * 6.2831853;
    const double sq = sqrt(1 - u1 * u1);
    const double dxn = sq * cos(th), dyn = u1, dzn = sq * sin(th);
    const double Rt = terrain_radius_at(t, coreR, d.cx + dxn * t.Rhi, d.cy + dyn * t.Rhi, d.cz + dzn * t.Rhi);
    dpt[a] = oceanR - Rt;
    const double rm = (Rt + oceanR) * 0.5;
    px[a] = d.cx + dxn * rm; py[a] = d.cy + dyn * rm; pz[a] = d.cz + dzn * rm;
  }
  __syncthreads();
  if (a == 0) {
    int pick = -1, used = 64;
    double bestD = -1;
    int best = -1;
    for (int k = 0; k < 64; k++) {
      if (dpt[k] > need) { pick = k; used = k + 1; break; }
      if (dpt[k] > bestD) { bestD = dpt[k]; best = k; }
    }
    if (pick < 0) pick = best;
    if (pick >= 0) { out[0] = px[pick]; out[1] = py[pick]; out[2] = pz[pick]; }
    else { out[0] = d.cx; out[1] = d.cy + oceanR; out[2] = d.cz; }
    out[3] = used;
  }
}
void launch_ocean_point(const Dims& d, const TerrainDev& t, double coreR, double oceanR, double need, uint32_t s0,
                        double* out, cudaStream_t s) {
  k_ocean_point<<<1, 64, 0, s>>>(d, t, coreR, oceanR, need, s0, out);
}
