// ws_frame.cu — per-frame passes: thermal tick (js/solver.js:2715-2994),
// evaporation (:3008-3125), phase changes (:3145-3281), frame-end rescue
// (:3496-3587), density splat (:3785-3820) and the FP64 reductions
// (marching-tets volume js/surface.js:66-177, census js/main.js:176-186,
// kinetic energy js/solver.js:3914-3921).
#include "ws_kernels.cuh"

// ------------------------------------------------------------ thermal: shadows + heating
// _heatShadowChunk, js/solver.js:2773-2918 — independent per particle.
__global__ void k_heat_shadow(Dims d, GridDev g, PartsDev P, TerrainDev t, HeatParams hp, double dt) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nP) return;
  const double dx = d.dx, cx = d.cx, cy = d.cy, cz = d.cz;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  const uint8_t* type = g.type;
  double lit = hp.hasSun ? 1 : 0;
  double PX = P.px[p], PY = P.py[p], PZ = P.pz[p];
  double dwx = PX - cx, dwy = PY - cy, dwz = PZ - cz;
  double dwl = sqrt(dwx * dwx + dwy * dwy + dwz * dwz); if (dwl == 0) dwl = 1e-9;
  double stpU = dx / dwl; int above = 0;
  for (int stU = 1; stU <= 4; stU++) {
    double qx = PX + dwx * stpU * stU, qy = PY + dwy * stpU * stU, qz = PZ + dwz * stpU * stU;
    int qi = jtrunc(over_dx(d, qx)), qj = jtrunc(over_dx(d, qy)), qk = jtrunc(over_dx(d, qz));
    if (qi < 0 || qj < 0 || qk < 0 || qi >= nx || qj >= ny || qk >= nz) break;
    if (type[((long long)qk * ny + qj) * nx + qi] != WS_FLUID) break;
    above++;
  }
  P.pDepth[p] = (uint8_t)above;
  if (hp.hasSun) {
    if (above >= 4) lit = 0;
    else {
      double lx = hp.sun[0] - PX, ly = hp.sun[1] - PY, lz = hp.sun[2] - PZ;
      double ld = sqrt(lx * lx + ly * ly + lz * lz); if (ld == 0) ld = 1e-9;
      double dxn = lx / ld, dyn = ly / ld, dzn = lz / ld;
      double ex = cx - PX, ey = cy - PY, ez = cz - PZ;
      double b = ex * dxn + ey * dyn + ez * dzn;
      if (t.has) {
        double d2c = ex * ex + ey * ey + ez * ez - b * b;
        if (b > 0 && d2c < t.Rlo2 * 0.96) lit = 0;
        else if (b > 0 || d2c < t.Rhi2 * 1.1) {
          double stp = dx * 1.5, mx = PX, my = PY, mz = PZ;
          double esc2 = (t.Rhi + 0.1) * (t.Rhi + 0.1);
          for (int st2 = 0; st2 < 26; st2++) {
            mx += dxn * stp; my += dyn * stp; mz += dzn * stp;
            double rex = mx - cx, rey = my - cy, rez = mz - cz;
            if (rex * rex + rey * rey + rez * rez > esc2) break;
            int ivx = jtrunc(over_dv(t, mx)); if (ivx < 0 || ivx >= t.n) break;
            int ivy = jtrunc(over_dv(t, my)); if (ivy < 0 || ivy >= t.n) break;
            int ivz = jtrunc(over_dv(t, mz)); if (ivz < 0 || ivz >= t.n) break;
            if (t.solid[((long long)ivz * t.n + ivy) * t.n + ivx]) { lit = 0; break; }
          }
        }
      } else if (b > 0) {
        double d2c2 = ex * ex + ey * ey + ez * ez - b * b;
        if (d2c2 < hp.coreR * hp.coreR) lit = 0;
      }
      if (lit != 0) {
        double od = 0, sx = PX, sy = PY, sz = PZ, half = dx;
        long long sj = nx + 1, sk = (long long)(ny + 1) * sj;
        for (int st = 0; st < 6 && st * half < 0.55; st++) {
          sx += dxn * half; sy += dyn * half; sz += dzn * half;
          int i0 = jtrunc(over_dx(d, sx)), j0 = jtrunc(over_dx(d, sy)), k0 = jtrunc(over_dx(d, sz));
          if (i0 < 0 || j0 < 0 || k0 < 0 || i0 >= nx || j0 >= ny || k0 >= nz) break;
          double vv = g.dens[k0 * sk + j0 * sj + i0];
          od += vv * half * 1.1;
          if (od > 3.5) break;
        }
        lit = od < 3.5 ? exp(-od) : 0;
      }
    }
  }
  P.pLight[p] = (float)lit;
  double T, pT = P.pT[p], Tamb = hp.Tamb, sunPow = hp.sunActivity / 3;
  int f = P.pflag[p];
  if (f == 2) {
    double amb = lit > 0.05 ? Tamb + 0.18 : 0.06, K = hp.hasSun ? 0.16 + (1 - lit) * 0.20 : 1.2;
    T = pT + (amb - pT) * K * dt; if (lit > 0) T += sunPow * 0.6 * lit * dt;
  } else if (f == 3) {
    double amb = lit > 0.05 ? Tamb + 0.18 : 0.06, K = hp.hasSun ? 0.10 + (1 - lit) * 0.12 : 0.9;
    T = pT + (amb - pT) * K * dt; if (lit > 0) T += sunPow * 0.35 * lit * dt;
  } else if (f == 4) {
    double amb = lit > 0.05 ? Tamb + 0.18 : 0.06, K = hp.hasSun ? 0.14 + (1 - lit) * 0.16 : 1.0;
    T = pT + (amb - pT) * K * dt; if (lit > 0) T += sunPow * 0.45 * lit * dt;
  } else {
    double amb = lit > 0.05 ? Tamb : 0;
    T = pT + (amb - pT) * (0.045 + (1 - lit) * hp.shadeCool) * dt; if (lit > 0) T += sunPow * lit * dt;
  }
  if (T > 1.15) T = 1.15; else if (T < 0) T = 0;
  P.pT[p] = (float)T;
}

// ------------------------------------------------------------ thermal: conduction
// Cell aggregates of _heatMeansSlice/_heatConductFlux/_heatApplySlice
// (:2921-2979) without a particle sort: counts and FP64 temperature sums per
// cell, then each cell gathers its six edge energies in the reference's
// accumulation order, then each particle applies its cell's update.
__device__ __forceinline__ long long heat_cell(const Dims& d, double x, double y, double z) {
  int gx = jtrunc(over_dx(d, x)); if (gx < 0) gx = 0; else if (gx >= d.nx) gx = d.nx - 1;
  int gy = jtrunc(over_dx(d, y)); if (gy < 0) gy = 0; else if (gy >= d.ny) gy = d.ny - 1;
  int gz = jtrunc(over_dx(d, z)); if (gz < 0) gz = 0; else if (gz >= d.nz) gz = d.nz - 1;
  return ((long long)gz * d.ny + gy) * d.nx + gx;
}
__global__ void k_heat_bin(Dims d, PartsDev P, int* __restrict__ cnt, double* __restrict__ sumT) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nP) return;
  long long c = heat_cell(d, P.px[p], P.py[p], P.pz[p]);
  atomicAdd(&cnt[c], 1);
  atomicAdd(&sumT[c], (double)P.pT[p]);
}
__global__ void k_heat_means(Dims d, const int* __restrict__ cnt, double* __restrict__ sumT) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= d.nCells) return;
  sumT[c] = cnt[c] ? sumT[c] / cnt[c] : 0.0;        // in place: sum -> mean
}
__global__ void k_heat_flux(Dims d, const int* __restrict__ cnt, const double* __restrict__ mean,
                            double* __restrict__ change, double alpha) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= d.nCells) return;
  int nc = cnt[c];
  if (!nc) return;
  int nx = d.nx, ny = d.ny, nz = d.nz; long long nxy = (long long)nx * ny;
  int i, j, k; cell_ijk(d, c, i, j, k);
  double ch = 0;
  // contributions as the neighbour of an earlier cell (:2961 "-="): c-nxy, c-nx, c-1
  if (k > 0 && cnt[c - nxy]) { int a = cnt[c - nxy]; ch -= alpha * (double)(a < nc ? a : nc) * (mean[c] - mean[c - nxy]); }
  if (j > 0 && cnt[c - nx]) { int a = cnt[c - nx]; ch -= alpha * (double)(a < nc ? a : nc) * (mean[c] - mean[c - nx]); }
  if (i > 0 && cnt[c - 1]) { int a = cnt[c - 1]; ch -= alpha * (double)(a < nc ? a : nc) * (mean[c] - mean[c - 1]); }
  // own edges along +x, +y, +z (:2961 "+=")
  if (i < nx - 1 && cnt[c + 1]) { int a = cnt[c + 1]; ch += alpha * (double)(nc < a ? nc : a) * (mean[c + 1] - mean[c]); }
  if (j < ny - 1 && cnt[c + nx]) { int a = cnt[c + nx]; ch += alpha * (double)(nc < a ? nc : a) * (mean[c + nx] - mean[c]); }
  if (k < nz - 1 && cnt[c + nxy]) { int a = cnt[c + nxy]; ch += alpha * (double)(nc < a ? nc : a) * (mean[c + nxy] - mean[c]); }
  change[c] = ch;
}
__global__ void k_heat_apply_convect(Dims d, PartsDev P, const int* __restrict__ cnt, const double* __restrict__ mean,
                                     const double* __restrict__ change, double alphaA, int conduct, double Tamb, double dt) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nP) return;
  double x = P.px[p], y = P.py[p], z = P.pz[p];
  float T = P.pT[p];
  if (conduct) {
    long long c = heat_cell(d, x, y, z);
    double deltaT = change[c] / cnt[c];
    T = (float)((double)T + alphaA * (mean[c] - (double)T) + deltaT);
    P.pT[p] = T;
  }
  if (P.pflag[p] != 0) return;                       // _heatConvectChunk :2982-2994
  double rx = x - d.cx, ry = y - d.cy, rz = z - d.cz;
  double rl = sqrt(rx * rx + ry * ry + rz * rz); if (rl == 0) rl = 1e-9;
  double ab = 3.0 * ((double)T - Tamb) * dt / rl;
  P.pvx[p] = (float)((double)P.pvx[p] + rx * ab);
  P.pvy[p] = (float)((double)P.pvy[p] + ry * ab);
  P.pvz[p] = (float)((double)P.pvz[p] + rz * ab);
}
void launch_heat(const Dims& d, const GridDev& g, const PartsDev& P, const TerrainDev& t, const HeatParams& hp,
                 double dt, int* cnt, double* sumT, double* change, cudaStream_t s) {
  if (P.nP <= 0) return;
  unsigned gp = grid_for(P.nP, 256), gc = grid_for(d.nCells, 256);
  k_heat_shadow<<<gp, 256, 0, s>>>(d, g, P, t, hp, dt);
  int conduct = hp.heatK > 0;
  if (conduct) {
    cudaMemsetAsync(cnt, 0, sizeof(int) * d.nCells, s);
    cudaMemsetAsync(sumT, 0, sizeof(double) * d.nCells, s);
    k_heat_bin<<<gp, 256, 0, s>>>(d, P, cnt, sumT);
    k_heat_means<<<gc, 256, 0, s>>>(d, cnt, sumT);
    double alpha = hp.heatK * dt * 0.15; if (alpha > 0.14) alpha = 0.14;
    k_heat_flux<<<gc, 256, 0, s>>>(d, cnt, sumT, change, alpha);
    k_heat_apply_convect<<<gp, 256, 0, s>>>(d, P, cnt, sumT, change, alpha, 1, hp.Tamb, dt);
  } else {
    k_heat_apply_convect<<<gp, 256, 0, s>>>(d, P, cnt, sumT, change, 0, 0, hp.Tamb, dt);
  }
}

// ------------------------------------------------------------ evaporation
// _evapChunk, js/solver.js:3028-3116. Candidates (surface-top liquid above
// the freezing point) are compacted in index order and walked as the
// reference's single _evS stream. With E ejections before it, candidate t
// (counted from the walk's start state s0) draws the state T^(t+1+6E)(s0),
// T the generator, each ejection taking six draws for its Box-Muller kick;
// it ejects when that draw u has u / 2^32 <= prob, i.e. u <= floor(prob 2^32).
// The walk is cut into windows of kEvW candidates. A window maps the
// ejection count before it to the count after it, monotonically; each window
// tabulates that map for a band of inputs around the expected count (the
// prefix sum of the probabilities), one warp per input, all windows in
// parallel; one warp then chains the windows through their tables (resolving
// a window directly when the count falls outside its band), and every window
// finally replays its own resolve to record its ejectors. A kick whose
// u1 < 1e-9 retry takes more than six draws (about one in 10^9) shifts every
// later position: the pass reports the first such ejection and the host starts
// a new pass after it.
__device__ __forceinline__ bool evap_candidate(const Dims& d, const GridDev& g, const PartsDev& P, int p,
                                               double freezeT, int& ci, int& cj, int& ck) {
  if (P.pflag[p] != 0) return false;
  double T = P.pT[p];
  if (T <= freezeT) return false;
  double PX = P.px[p], PY = P.py[p], PZ = P.pz[p];
  int i = jtrunc(over_dx(d, PX)), j = jtrunc(over_dx(d, PY)), k = jtrunc(over_dx(d, PZ));
  if (i < 1) i = 1; else if (i > d.nx - 2) i = d.nx - 2;
  if (j < 1) j = 1; else if (j > d.ny - 2) j = d.ny - 2;
  if (k < 1) k = 1; else if (k > d.nz - 2) k = d.nz - 2;
  if (g.type[((long long)k * d.ny + j) * d.nx + i] != WS_FLUID) return false;
  double ex = PX - d.cx, ey = PY - d.cy, ez = PZ - d.cz;
  double el = sqrt(ex * ex + ey * ey + ez * ez); if (el == 0) el = 1e-9;
  int ui = jtrunc(over_dx(d, PX + ex / el * d.dx)), uj = jtrunc(over_dx(d, PY + ey / el * d.dx)), uk = jtrunc(over_dx(d, PZ + ez / el * d.dx));
  if (ui < 0 || uj < 0 || uk < 0 || ui >= d.nx || uj >= d.ny || uk >= d.nz) return false;
  if (g.type[((long long)uk * d.ny + uj) * d.nx + ui] == WS_FLUID) return false;
  ci = i; cj = j; ck = k;
  return true;
}
__global__ void k_evap_flags(Dims d, GridDev g, PartsDev P, double freezeT, uint8_t* __restrict__ cand) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nP) return;
  int i, j, k;
  cand[p] = evap_candidate(d, g, P, p, freezeT, i, j, k) ? 1 : 0;
}
__device__ __forceinline__ double ev_gauss(uint32_t& s) {
  double u1;
  do { s = lcg_next(s); u1 = s / 4294967296.0; } while (u1 < 1e-9);
  s = lcg_next(s);
  return sqrt(-2 * log(u1)) * cos(6.283185306 * (s / 4294967296.0));
}
uint32_t evap_kick_end(uint32_t s) {             // the stream after a kick drawn from decision state s
  for (int g = 0; g < 3; g++) {
    do { s = lcg_next(s); } while (s < 5u);       // u1 = s / 2^32 < 1e-9 exactly when s < 5
    s = lcg_next(s);
  }
  return s;
}
// Six steps of the _evS generator (x -> 1664525 x + 1013904223 mod 2^32) as one affine map.
constexpr uint32_t lcg_pow_a(int n) { return n == 0 ? 1u : 1664525u * lcg_pow_a(n - 1); }
constexpr uint32_t lcg_pow_c(int n) { return n == 0 ? 0u : 1664525u * lcg_pow_c(n - 1) + 1013904223u; }
constexpr uint32_t kLcg6A = lcg_pow_a(6), kLcg6C = lcg_pow_c(6);
constexpr double kEvapC = 3.5, kEvapTCap = 1.15;   // EVAP_STEEPNESS and T_CAP, js/solver.js:3040-3041
constexpr int kEvW = 4096;                       // candidates per window
constexpr int kEvKMax = 1024;                    // widest band of tabulated inputs per window
__device__ __forceinline__ void lcg_affine(uint32_t k, uint32_t& A, uint32_t& C) {   // T^k(x) = A x + C
  uint32_t a = 1664525u, c = 1013904223u;
  A = 1u; C = 0u;
  while (k) { if (k & 1u) { A = A * a; C = C * a + c; } c = c * (a + 1u); a = a * a; k >>= 1; }
}
// The candidate ejects when its draw u satisfies u <= thr (thr = -1: never;
// 2^32: always, prob >= 1 or NaN as in !(rnd > prob)).
__global__ void k_evap_thr(const PartsDev P, double freezeT, double rate, double dt, const int* __restrict__ list,
                           const int* __restrict__ nCp, long long* __restrict__ thr) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= *nCp) return;
  double prob = rate * dt * exp(kEvapC * ((double)P.pT[list[t]] - freezeT));
  long long v;
  if (!(prob < 1)) v = 4294967296ll;
  else if (prob < 0) v = -1;
  else v = (long long)floor(prob * 4294967296.0);
  thr[t] = v;
}
// One warp resolves a window of n candidates entering with Ein ejections:
// b[j] = T^(j'+1)(s0) for the window's j-th candidate (j' its index in the
// pass), so its draw after E ejections is T^(6E)(b[j]). Returns the count
// after the window; emit(j, E, u) runs on the lane of each ejector.
template <class Emit>
__device__ __forceinline__ int ev_resolve(const uint32_t* b, const long long* thr, int n, int Ein, Emit emit) {
  const int lane = threadIdx.x & 31;
  uint32_t A, C;
  lcg_affine(6u * (uint32_t)Ein, A, C);
  int E = Ein, i = 0;
  while (i < n) {
    const int idx = i + lane;
    uint32_t u = 0;
    bool hit = false;
    if (idx < n) { u = A * b[idx] + C; hit = (long long)u <= thr[idx]; }
    const unsigned bal = __ballot_sync(0xffffffffu, hit);
    if (!bal) { i += 32; continue; }
    const int f = __ffs(bal) - 1;
    if (lane == f) emit(idx, E, u);
    E++; i += f + 1;
    C = kLcg6A * C + kLcg6C; A = kLcg6A * A;
  }
  return E;
}
__device__ __forceinline__ int ev_windows(int nC, int t0) { return nC > t0 ? (nC - t0 + kEvW - 1) / kEvW : 0; }
__global__ void __launch_bounds__(256) k_evap_wsum(const long long* __restrict__ thr, const int* __restrict__ nCp,
                                                   int t0, double* __restrict__ wsum) {
  __shared__ double red[8];
  const int nC = *nCp, w = blockIdx.x;
  if (w >= ev_windows(nC, t0)) return;
  const int lo = t0 + w * kEvW, hi = min(nC, lo + kEvW);
  double acc = 0;
  for (int t = lo + (int)threadIdx.x; t < hi; t += blockDim.x) {
    const long long v = thr[t];
    acc += v < 0 ? 0.0 : v >= 4294967296ll ? 1.0 : (double)v * (1.0 / 4294967296.0);
  }
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0;
    for (int k = 0; k < 8; k++) tot += red[k];
    wsum[w] = tot;
  }
}
// Band origins: L[w] = floor(expected ejections before window w) - K/2, K set
// from the expected total (eight standard deviations of a Poisson count, + 64).
__global__ void __launch_bounds__(1024) k_evap_band(const double* __restrict__ wsum, const int* __restrict__ nCp,
                                                    int t0, int* __restrict__ L, DevStatus* st) {
  __shared__ double red[32];
  __shared__ double sTot;
  const int nW = ev_windows(*nCp, t0);
  const int tid = (int)threadIdx.x, lane = tid & 31, wid = tid >> 5;
  double v = 0;
  for (int w = tid; w < nW; w += 1024) v += wsum[w];
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (lane == 0) red[wid] = v;
  __syncthreads();
  if (tid == 0) { double tot = 0; for (int k = 0; k < 32; k++) tot += red[k]; sTot = tot; }
  __syncthreads();
  int keff = ((int)(8.0 * sqrt(sTot) + 64.0) + 31) & ~31;
  keff = keff < 64 ? 64 : keff > kEvKMax ? kEvKMax : keff;
  double carry = 0;
  for (int c0 = 0; c0 < nW; c0 += 1024) {
    __syncthreads();                              // red[] and sTot of the previous chunk are consumed
    const int w = c0 + tid;
    const double x = w < nW ? wsum[w] : 0.0;
    double inc = x;
    for (int o = 1; o < 32; o <<= 1) { double y = __shfl_up_sync(0xffffffffu, inc, o); if (lane >= o) inc += y; }
    if (lane == 31) red[wid] = inc;
    __syncthreads();
    if (wid == 0) {
      double r = red[lane], ri = r;
      for (int o = 1; o < 32; o <<= 1) { double y = __shfl_up_sync(0xffffffffu, ri, o); if (lane >= o) ri += y; }
      red[lane] = ri - r;                         // exclusive warp offsets
      if (lane == 31) sTot = ri;
    }
    __syncthreads();
    const double excl = carry + red[wid] + inc - x;
    if (w < nW) { const int c = (int)floor(excl) - keff / 2; L[w] = c < 0 ? 0 : c; }
    carry += sTot;
  }
  if (tid == 0) { st->evKeff = keff; st->evIrr = ~0ull; st->evNC = *nCp; }
}
// Each window: its candidates' base states and thresholds in shared memory,
// then one warp per tabulated input.
__global__ void __launch_bounds__(1024) k_evap_table(const long long* __restrict__ thr, const int* __restrict__ nCp,
                                                     int t0, const uint32_t* __restrict__ sStart,
                                                     const int* __restrict__ L, const DevStatus* __restrict__ st,
                                                     uint32_t* __restrict__ bOut, unsigned short* __restrict__ table) {
  __shared__ uint32_t sb[kEvW];
  __shared__ long long sthr[kEvW];
  const int nC = *nCp, w = blockIdx.x;
  if (w >= ev_windows(nC, t0)) return;
  const int lo = t0 + w * kEvW, n = min(kEvW, nC - lo);
  const uint32_t s0 = *sStart;
  for (int j = (int)threadIdx.x; j < n; j += blockDim.x) {
    const uint32_t bj = lcg_jump(s0, (uint32_t)(lo - t0 + j + 1));
    sb[j] = bj; bOut[lo + j] = bj;
    sthr[j] = thr[lo + j];
  }
  __syncthreads();
  const int keff = st->evKeff, Lw = L[w];
  for (int k = (int)(threadIdx.x >> 5); k < keff; k += (int)(blockDim.x >> 5)) {
    const int eo = ev_resolve(sb, sthr, n, Lw + k, [](int, int, uint32_t) {});
    if ((threadIdx.x & 31) == 0) table[(size_t)w * kEvKMax + k] = (unsigned short)(eo - (Lw + k));
  }
}
// One warp: the ejection count entering every window.
__global__ void __launch_bounds__(32) k_evap_chain(const int* __restrict__ nCp, int t0, const int* __restrict__ L,
                                                   const unsigned short* __restrict__ table,
                                                   const uint32_t* __restrict__ b, const long long* __restrict__ thr,
                                                   const uint32_t* __restrict__ sStart, int* __restrict__ Ew,
                                                   DevStatus* st) {
  const int nC = *nCp, nW = ev_windows(nC, t0), keff = st->evKeff;
  int E = 0;
  int Lnext = nW > 0 ? L[0] : 0;
  for (int w = 0; w < nW; w++) {
    const int Lw = Lnext;
    if (w + 1 < nW) Lnext = L[w + 1];
    if (threadIdx.x == 0) Ew[w] = E;
    const int rel = E - Lw;
    if (rel >= 0 && rel < keff) {
      E += table[(size_t)w * kEvKMax + rel];
    } else {
      const int lo = t0 + w * kEvW;
      E = ev_resolve(b + lo, thr + lo, min(kEvW, nC - lo), E, [](int, int, uint32_t) {});
    }
  }
  if (threadIdx.x == 0) {
    st->evNEj = E;
    st->evSEnd = lcg_jump(*sStart, (uint32_t)(nC > t0 ? nC - t0 : 0) + 6u * (uint32_t)E);
  }
}
// One warp per window: replay its resolve and record each ejector (particle and decision state).
__global__ void k_evap_emit(const int* __restrict__ nCp, int t0, const uint32_t* __restrict__ b,
                            const long long* __restrict__ thr, const int* __restrict__ Ew, const int* __restrict__ list,
                            int eoff, int* __restrict__ ejP, uint32_t* __restrict__ ejS, DevStatus* st) {
  const int nC = *nCp;
  const int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (w >= ev_windows(nC, t0)) return;          // uniform over the warp
  const int lo = t0 + w * kEvW;
  ev_resolve(b + lo, thr + lo, min(kEvW, nC - lo), Ew[w], [&](int j, int E, uint32_t u) {
    ejP[eoff + E] = list[lo + j];
    ejS[eoff + E] = u;
    // Regular kick: its three u1 draws (1, 3 and 5 after the decision) have states >= 5.
    const uint32_t s1 = lcg_next(u), s3 = lcg_next(lcg_next(s1)), s5 = lcg_next(lcg_next(s3));
    if (s1 < 5u || s3 < 5u || s5 < 5u)
      atomicMin(&st->evIrr, ((unsigned long long)(unsigned)E << 32) | (unsigned)(lo - t0 + j));
  });
}
// :3083-3113 for one ejection, its kick drawn from the recorded stream state.
__global__ void k_evap_apply(Dims d, GridDev g, PartsDev P, double freezeT, const int* __restrict__ ejP,
                             const uint32_t* __restrict__ ejS, int nEj) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nEj) return;
  const int p = ejP[e];
  int i, j, k;
  evap_candidate(d, g, P, p, freezeT, i, j, k);
  const double T = P.pT[p];
  double tau = (T - freezeT) / (kEvapTCap - freezeT);
  if (tau < 0) tau = 0; else if (tau > 1) tau = 1;
  const double sig = 0.30 + 0.32 * sqrt(tau);
  uint32_t sl = ejS[e];
  double kx = sig * ev_gauss(sl); double ky = sig * ev_gauss(sl); double kz = sig * ev_gauss(sl);
  P.pflag[p] = 2; P.pAir[p] = 0.f;
  double PX = P.px[p], PY = P.py[p], PZ = P.pz[p];
  double ex2 = PX - d.cx, ey2 = PY - d.cy, ez2 = PZ - d.cz;
  double el2 = ex2 * ex2 + ey2 * ey2 + ez2 * ez2;
  double elL = sqrt(el2); if (elL == 0) elL = 1e-9;
  double kUp = (kx * ex2 + ky * ey2 + kz * ez2) / el2;
  if (kUp < 0) { kx -= 2 * kUp * ex2 / elL; ky -= 2 * kUp * ey2 / elL; kz -= 2 * kUp * ez2 / elL; }
  int nx = d.nx, ny = d.ny;
  double guS = g.vel[((long long)k * ny + j) * (nx + 1) + i];
  double gvS = g.vel[d.uN + ((long long)k * (ny + 1) + j) * nx + i];
  double gwS = g.vel[d.uN + d.vN + ((long long)k * ny + j) * nx + i];
  double nl2 = 1 / el2;
  double vN = ((double)P.pvx[p] * ex2 + (double)P.pvy[p] * ey2 + (double)P.pvz[p] * ez2) * nl2;
  double gN = (guS * ex2 + gvS * ey2 + gwS * ez2) * nl2;
  P.pvx[p] = (float)(vN * ex2 + (guS - gN * ex2) + kx);
  P.pvy[p] = (float)(vN * ey2 + (gvS - gN * ey2) + ky);
  P.pvz[p] = (float)(vN * ez2 + (gwS - gN * ez2) + kz);
}
static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
static size_t ev_max_windows(int cap) { return (size_t)(cap + kEvW - 1) / kEvW + 1; }
size_t evaporation_scratch_bytes(int cap) {
  const size_t c = (size_t)cap, nw = ev_max_windows(cap);
  return align256(8 * c) + 4 * align256(4 * c) + align256(8 * nw) + 2 * align256(4 * nw) + align256(2 * kEvKMax * nw);
}
EvapScratch evap_carve(void* base, int cap) {
  const size_t c = (size_t)cap, nw = ev_max_windows(cap);
  char* q = (char*)base; EvapScratch e;
  e.thr = (long long*)q; q += align256(8 * c);
  e.b = (uint32_t*)q; q += align256(4 * c);
  e.ejP = (int*)q; q += align256(4 * c);
  e.ejS = (uint32_t*)q; q += align256(4 * c);
  q += align256(4 * c);                           // reserved
  e.wsum = (double*)q; q += align256(8 * nw);
  e.L = (int*)q; q += align256(4 * nw);
  e.Ew = (int*)q; q += align256(4 * nw);
  e.table = (unsigned short*)q;
  return e;
}
void launch_evap_prepare(const Dims& d, const GridDev& g, const PartsDev& P, double freezeT, double rate, double dt,
                         uint8_t* cand, int* blockCounts, int* list, int* nC, const EvapScratch& es, cudaStream_t s) {
  const int gp = grid_for(P.nP, 256);
  k_evap_flags<<<gp, 256, 0, s>>>(d, g, P, freezeT, cand);
  launch_compact(cand, P.nP, 2, blockCounts, list, nC, s);
  k_evap_thr<<<gp, 256, 0, s>>>(P, freezeT, rate, dt, list, nC, es.thr);
}
void launch_evap_pass(int nP, const int* list, const int* nC, const EvapScratch& es, int t0, int eoff,
                      const uint32_t* sStart, DevStatus* st, cudaStream_t s) {
  const int nw = (int)ev_max_windows(nP);
  k_evap_wsum<<<nw, 256, 0, s>>>(es.thr, nC, t0, es.wsum);
  k_evap_band<<<1, 1024, 0, s>>>(es.wsum, nC, t0, es.L, st);
  k_evap_table<<<nw, 1024, 0, s>>>(es.thr, nC, t0, sStart, es.L, st, es.b, es.table);
  k_evap_chain<<<1, 32, 0, s>>>(nC, t0, es.L, es.table, es.b, es.thr, sStart, es.Ew, st);
  k_evap_emit<<<(nw + 3) / 4, 128, 0, s>>>(nC, t0, es.b, es.thr, es.Ew, list, eoff, es.ejP, es.ejS, st);
}
void launch_evap_apply(const Dims& d, const GridDev& g, const PartsDev& P, double freezeT, const EvapScratch& es,
                       int nEj, cudaStream_t s) {
  if (nEj > 0) k_evap_apply<<<grid_for(nEj, 256), 256, 0, s>>>(d, g, P, freezeT, es.ejP, es.ejS, nEj);
}

// ------------------------------------------------------------ phase changes
// _updatePhaseChanges, js/solver.js:3152-3281: steam counts per cell
// (integer atomics, exact), then independent per-particle transitions.
__device__ __forceinline__ long long clamp_cell(const Dims& d, double x, double y, double z, int& i, int& j, int& k) {
  i = jtrunc(over_dx(d, x)); j = jtrunc(over_dx(d, y)); k = jtrunc(over_dx(d, z));
  if (i < 0) i = 0; else if (i >= d.nx) i = d.nx - 1;
  if (j < 0) j = 0; else if (j >= d.ny) j = d.ny - 1;
  if (k < 0) k = 0; else if (k >= d.nz) k = d.nz - 1;
  return ((long long)k * d.ny + j) * d.nx + i;
}
__global__ void k_steam_count(Dims d, PartsDev P, int* __restrict__ cnt) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nP || P.pflag[p] != 2) return;
  int i, j, k;
  atomicAdd(&cnt[clamp_cell(d, P.px[p], P.py[p], P.pz[p], i, j, k)], 1);
}
__device__ __forceinline__ uint32_t js_mul_u32(double a, double b) {
  double m = fmod(a * b, 4294967296.0); if (m < 0) m += 4294967296.0;
  return (uint32_t)m;
}
__device__ __forceinline__ uint32_t spin_hash(uint32_t a, uint32_t b, uint32_t c) {   // :3145-3150
  uint32_t s = a ^ js_mul_u32(b, 2654435769.0) ^ js_mul_u32(c, 2246822507.0) ^ js_mul_u32(1370176631.0, 3266489909.0);
  s = lcg_next(s);
  s ^= s >> 13; s = js_mul_u32(s, 1540483477.0); s ^= s >> 15;
  return s;
}
__global__ void k_phase_update(Dims d, GridDev g, PartsDev P, PhaseParams pp, const int* __restrict__ cnt) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nP) return;
  const uint8_t* type = g.type;
  int nx = d.nx, ny = d.ny, nz = d.nz; long long nxy = (long long)nx * ny;
  int f = P.pflag[p], i, j, k;
  double T = P.pT[p];
  if (f == 0) {
    if (T <= pp.snowT && T > 1e-3) {
      long long cB = clamp_cell(d, P.px[p], P.py[p], P.pz[p], i, j, k);
      bool atSurf = (k > 0 && type[cB - nxy] != WS_FLUID) || (k < nz - 1 && type[cB + nxy] != WS_FLUID) ||
                    (j > 0 && type[cB - nx] != WS_FLUID) || (j < ny - 1 && type[cB + nx] != WS_FLUID) ||
                    (i > 0 && type[cB - 1] != WS_FLUID) || (i < nx - 1 && type[cB + 1] != WS_FLUID);
      if (atSurf) { P.pflag[p] = 5; P.pvx[p] = P.pvy[p] = P.pvz[p] = 0.f; P.pAir[p] = 1.f; }
    }
  } else if (f == 5) {
    if (T >= pp.meltT) {
      long long c = clamp_cell(d, P.px[p], P.py[p], P.pz[p], i, j, k);
      P.pflag[p] = type[c] == WS_FLUID ? 0 : 4;
      P.pAir[p] = 0.f; P.pWx[p] = P.pWy[p] = P.pWz[p] = 0.f;
    }
  } else if (T > 1e-3) {
    if (f == 2) {
      if (T <= pp.rainT && (double)P.pAir[p] >= pp.rainLiftAge) {
        P.pflag[p] = 4; P.pAir[p] = 0.f; P.pvx[p] = P.pvy[p] = P.pvz[p] = 0.f; P.pWx[p] = P.pWy[p] = P.pWz[p] = 0.f;
        f = 4;
      } else if (T <= pp.cloudT) {
        double rx = (double)P.px[p] - d.cx, ry = (double)P.py[p] - d.cy, rz = (double)P.pz[p] - d.cz;
        if (sqrt(rx * rx + ry * ry + rz * rz) >= pp.cloudBase) {
          i = jtrunc(over_dx(d, P.px[p])); j = jtrunc(over_dx(d, P.py[p])); k = jtrunc(over_dx(d, P.pz[p]));
          int i0 = i > 0 ? i - 1 : 0, i1 = i < nx - 1 ? i + 1 : nx - 1;
          int j0 = j > 0 ? j - 1 : 0, j1 = j < ny - 1 ? j + 1 : ny - 1;
          int k0 = k > 0 ? k - 1 : 0, k1 = k < nz - 1 ? k + 1 : nz - 1;
          double sum = 0;
          for (int kk = k0; kk <= k1; kk++) for (int jj = j0; jj <= j1; jj++) {
            long long row = ((long long)kk * ny + jj) * nx;
            for (int ii = i0; ii <= i1; ii++) sum += cnt[row + ii];
          }
          if (sum / 27 >= pp.cloudP) { P.pflag[p] = 3; P.pAir[p] = 0.f; f = 3; }
        }
      }
    } else if (f == 3) {
      if (T >= pp.cloudT + 0.05) { P.pflag[p] = 2; f = 2; }
    } else if ((f == 1 || f == 4) && T <= pp.snowT) {   // spray and rain freeze (:3253)
      P.pflag[p] = 5; P.pvx[p] = P.pvy[p] = P.pvz[p] = 0.f; P.pAir[p] = 0.f; P.pWx[p] = P.pWy[p] = P.pWz[p] = 0.f;
    }
  }
}
// spin bookkeeping (:3259-3280), a separate pass over the final flags
__global__ void k_phase_spin(PartsDev P, uint32_t tick, double dt) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nP) return;
  int f = P.pflag[p];
  if (f != 2 && f != 3) return;
  float wx = P.pWx[p], wy = P.pWy[p], wz = P.pWz[p];
  if (f == 2 && P.pAir[p] <= 1e-6f && wx == 0.f && wy == 0.f && wz == 0.f) {
    uint32_t sd = 0x51ab3c77u;
    double h1 = spin_hash(sd, (uint32_t)p, tick) / 4294967296.0;
    double h2 = spin_hash(sd + 1, (uint32_t)p, tick) / 4294967296.0;
    double h3 = spin_hash(sd + 2, (uint32_t)p, tick) / 4294967296.0;
    double zz = 2 * h2 - 1, rr = sqrt(dmax(0, 1 - zz * zz)), th = 6.283185306 * h1;
    double Tp = P.pT[p]; if (!(Tp > 0.05)) Tp = 0.05; else if (Tp > 1.15) Tp = 1.15;
    double wSpd = 3.0 * sqrt(Tp) * (0.5 + h3);
    wx = (float)(rr * cos(th) * wSpd); wy = (float)(zz * wSpd); wz = (float)(rr * sin(th) * wSpd);
  }
  double wm = sqrt((double)wx * wx + (double)wy * wy + (double)wz * wz);
  if (wm > 1e-6) P.pPh[p] = (float)((double)P.pPh[p] + wm * dt);
  double damp = dmax(0, 1 - 0.12 * dt);
  P.pWx[p] = (float)(wx * damp); P.pWy[p] = (float)(wy * damp); P.pWz[p] = (float)(wz * damp);
}
void launch_phase(const Dims& d, const GridDev& g, const PartsDev& P, const PhaseParams& pp, int* cnt, cudaStream_t s) {
  if (P.nP <= 0) return;
  cudaMemsetAsync(cnt, 0, sizeof(int) * d.nCells, s);
  unsigned gp = grid_for(P.nP, 256);
  k_steam_count<<<gp, 256, 0, s>>>(d, P, cnt);
  k_phase_update<<<gp, 256, 0, s>>>(d, g, P, pp, cnt);
  if (pp.spinOn && pp.dt > 0) k_phase_spin<<<gp, 256, 0, s>>>(P, pp.tick, pp.dt);
}

// ------------------------------------------------------------ frame-end rescue
// _pushSurfaceChunk, js/solver.js:3496-3587 — independent per particle.
__global__ void k_push_surface(Dims d, GridDev g, PartsDev P, TerrainDev t, double oceanR, double coreR, double atmosphereH) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nP || !t.has) return;
  const double cx = d.cx, cy = d.cy, cz = d.cz, dx = d.dx;
  double x = P.px[p], y = P.py[p], z = P.pz[p];
  float fvx = P.pvx[p], fvy = P.pvy[p], fvz = P.pvz[p];
  double ex = x - cx, ey = y - cy, ez = z - cz;
  double er = sqrt(ex * ex + ey * ey + ez * ez); if (er == 0) er = 1e-9;
  bool fixed = false, rockFixed = false, velChanged = false;
  double outer = d.domainR - dx * 0.02;
  double skyHi = oceanR + atmosphereH - 1e-3 * dx;
  if (er > skyHi) {
    x = cx + ex / er * skyHi; y = cy + ey / er * skyHi; z = cz + ez / er * skyHi;
    double outward = ((double)fvx * ex + (double)fvy * ey + (double)fvz * ez) / er;
    if (outward > 0) { fvx = (float)(fvx - ex / er * outward); fvy = (float)(fvy - ey / er * outward); fvz = (float)(fvz - ez / er * outward); velChanged = true; }
    ex = x - cx; ey = y - cy; ez = z - cz; er = skyHi;
    fixed = true;
  }
  if (er <= d.domainR && rock_cell_at(d, g.staticTypes, x, y, z)) {
    rockFixed = true;
    int tries = 0;
    while (rock_cell_at(d, g.staticTypes, x, y, z) && tries < d.nx * 2) {
      x += ex / er * dx * 0.5; y += ey / er * dx * 0.5; z += ez / er * dx * 0.5; tries++;
    }
    double exR = x - cx, eyR = y - cy, ezR = z - cz;
    double erR = sqrt(exR * exR + eyR * eyR + ezR * ezR); if (erR == 0) erR = 1e-9;
    double wantR = terrain_radius_at(t, coreR, x, y, z) + dx * 0.06;
    if (erR > wantR) { x = cx + exR / erR * wantR; y = cy + eyR / erR * wantR; z = cz + ezR / erR * wantR; }
    int kR = 0;
    while (rock_cell_at(d, g.staticTypes, x, y, z) && kR < 4) {
      x += exR / erR * dx * 0.5; y += eyR / erR * dx * 0.5; z += ezR / erR * dx * 0.5; kR++;
    }
    fixed = true;
  } else if (P.pflag[p] == 0 && er <= d.domainR) {
    double Rt = terrain_radius_at(t, coreR, x, y, z);
    if (er < Rt - dx * 0.5) {
      rockFixed = true;
      x = cx + ex / er * (Rt + dx * 0.05); y = cy + ey / er * (Rt + dx * 0.05); z = cz + ez / er * (Rt + dx * 0.05);
      int t2 = 0;
      while (rock_cell_at(d, g.staticTypes, x, y, z) && t2 < 8) {
        x += ex / er * dx * 0.5; y += ey / er * dx * 0.5; z += ez / er * dx * 0.5; t2++;
      }
      fixed = true;
    }
  }
  double finalR = sqrt((x - cx) * (x - cx) + (y - cy) * (y - cy) + (z - cz) * (z - cz));
  double capR = P.pflag[p] == 0 ? outer : skyHi;
  if (finalR > capR) {
    x = cx + (x - cx) * capR / finalR; y = cy + (y - cy) * capR / finalR; z = cz + (z - cz) * capR / finalR;
    fixed = true;
  }
  if (fixed) {
    P.px[p] = (float)x; P.py[p] = (float)y; P.pz[p] = (float)z;
    double vr = ((double)fvx * ex + (double)fvy * ey + (double)fvz * ez) / er;
    if (rockFixed && vr < 0) { fvx = (float)(fvx - ex / er * vr); fvy = (float)(fvy - ey / er * vr); fvz = (float)(fvz - ez / er * vr); velChanged = true; }
  }
  if (velChanged) { P.pvx[p] = fvx; P.pvy[p] = fvy; P.pvz[p] = fvz; }
}
void launch_push_surface(const Dims& d, const GridDev& g, const PartsDev& P, const TerrainDev& t,
                         double oceanR, double coreR, double atmosphereH, cudaStream_t s) {
  if (P.nP <= 0) return;
  k_push_surface<<<grid_for(P.nP, 256), 256, 0, s>>>(d, g, P, t, oceanR, coreR, atmosphereH);
}

// ------------------------------------------------------------ density splat
// _splatInto, js/solver.js:3792-3820 (float atomics on the corner lattice)
__global__ void k_splat(Dims d, GridDev g, PartsDev P, double spacing) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nP || P.pflag[p] != 0) return;
  double dx = d.dx, r = 1.6 * spacing, r2 = r * r;
  long long sj = d.nx + 1, sk = (long long)(d.ny + 1) * sj;
  double X = P.px[p], Y = P.py[p], Z = P.pz[p];
  double fi = floor(over_dx(d, X)), fj = floor(over_dx(d, Y)), fk = floor(over_dx(d, Z));
  int i0 = fi < 0 ? 0 : (fi > d.nx - 1 ? d.nx - 1 : (int)fi);
  int j0 = fj < 0 ? 0 : (fj > d.ny - 1 ? d.ny - 1 : (int)fj);
  int k0 = fk < 0 ? 0 : (fk > d.nz - 1 ? d.nz - 1 : (int)fk);
  double fx = X - i0 * dx, fy = Y - j0 * dx, fz = Z - k0 * dx;
  for (int kk = 0; kk < 2; kk++) {
    double czz = kk == 0 ? fz : fz - dx;
    for (int jj = 0; jj < 2; jj++) {
      double cyy = jj == 0 ? fy : fy - dx;
      for (int ii = 0; ii < 2; ii++) {
        double cxx = ii == 0 ? fx : fx - dx;
        double d2 = cxx * cxx + cyy * cyy + czz * czz;
        if (d2 >= r2) continue;
        double ww = 1 - d2 / r2; ww = ww * ww;
        atomicAdd(&g.dens[(k0 + kk) * sk + (j0 + jj) * sj + (i0 + ii)], (float)ww);
      }
    }
  }
}
void launch_splat(const Dims& d, const GridDev& g, const PartsDev& P, double spacing, cudaStream_t s) {
  long long nd = (long long)(d.nx + 1) * (d.ny + 1) * (d.nz + 1);
  cudaMemsetAsync(g.dens, 0, sizeof(float) * nd, s);
  if (P.nP <= 0) return;
  k_splat<<<grid_for(P.nP, 256), 256, 0, s>>>(d, g, P, spacing);
}

// ------------------------------------------------------------ marching-tets volume (FP64)
__constant__ int c_corners[8][3] = { {0,0,0},{1,0,0},{1,1,0},{0,1,0},{0,0,1},{1,0,1},{1,1,1},{0,1,1} };
__constant__ int c_tets[6][4] = { {0,5,1,6},{0,1,2,6},{0,2,3,6},{0,3,7,6},{0,7,4,6},{0,4,5,6} };
__constant__ int c_edges[6][2] = { {0,1},{1,2},{2,0},{0,3},{1,3},{2,3} };
__constant__ int c_ntri[16] = { 0,1,1,2,1,2,2,1,1,2,2,1,2,1,1,0 };
__constant__ int c_cases[16][2][3] = {
  {{0,0,0},{0,0,0}}, {{0,2,3},{0,0,0}}, {{0,1,4},{0,0,0}}, {{2,3,4},{2,4,1}},
  {{2,1,5},{0,0,0}}, {{0,3,5},{0,5,1}}, {{0,4,5},{0,5,2}}, {{3,5,4},{0,0,0}},
  {{3,4,5},{0,0,0}}, {{0,2,5},{0,5,4}}, {{0,1,5},{0,5,3}}, {{2,1,5},{0,0,0}},
  {{2,1,4},{2,4,3}}, {{0,1,4},{0,0,0}}, {{0,2,3},{0,0,0}}, {{0,0,0},{0,0,0}} };
// One cell's signed tet-mesh volume contribution and vertex count (the
// per-cell body of MarchingTetrahedra.build, js/surface.js:80-171).
// one cell of MarchingTetrahedra.build (js/surface.js:66-177): its signed
// volume, its vertex count and, when pos/nrm are given, its vertices
// (positions and gradient normals as float, 3 per vertex) from index base
// dxPow2: dx is a power of two, so the central differences' division by 2 dx
// is the exact product with r2dx = 1 / (2 dx) (see is_pow2)
__device__ double mt_cell(const float* __restrict__ dens, int nx, int ny, int nz, double dx, bool dxPow2, double r2dx,
                          double iso, int i, int j, int k, int& verts, float* pos = nullptr, float* nrm = nullptr,
                          long long base = 0) {
  long long sj = nx + 1, sk = (long long)(ny + 1) * sj;
  double cv[8], gx[8], gy[8], gz[8], minv = 1e300, maxv = -1e300;
  verts = 0;
  for (int c = 0; c < 8; c++) {
    double val = dens[(k + c_corners[c][2]) * sk + (j + c_corners[c][1]) * sj + (i + c_corners[c][0])];
    cv[c] = val; if (val < minv) minv = val; if (val > maxv) maxv = val;
  }
  if (maxv < iso || minv > iso) return 0;
  for (int c = 0; c < 8; c++) {
    int ci = i + c_corners[c][0], cj = j + c_corners[c][1], ck = k + c_corners[c][2];
    int ip = ci + 1 < nx ? ci + 1 : nx, im = ci - 1 > 0 ? ci - 1 : 0;
    int jp = cj + 1 < ny ? cj + 1 : ny, jm = cj - 1 > 0 ? cj - 1 : 0;
    int kp = ck + 1 < nz ? ck + 1 : nz, km = ck - 1 > 0 ? ck - 1 : 0;
    const double ddx = (double)dens[ck * sk + cj * sj + ip] - (double)dens[ck * sk + cj * sj + im];
    const double ddy = (double)dens[ck * sk + jp * sj + ci] - (double)dens[ck * sk + jm * sj + ci];
    const double ddz = (double)dens[kp * sk + cj * sj + ci] - (double)dens[km * sk + cj * sj + ci];
    if (dxPow2) { gx[c] = ddx * r2dx; gy[c] = ddy * r2dx; gz[c] = ddz * r2dx; }
    else { gx[c] = ddx / (2 * dx); gy[c] = ddy / (2 * dx); gz[c] = ddz / (2 * dx); }
  }
  double vol = 0;
  for (int t = 0; t < 6; t++) {
    int code = 0;
    for (int c = 0; c < 4; c++) if (cv[c_tets[t][c]] > iso) code |= 1 << c;
    int ntri = c_ntri[code];
    for (int e = 0; e < ntri; e++) {
      double P3[3][3], N3[3][3];
      for (int vi = 0; vi < 3; vi++) {
        int ed = c_cases[code][e][vi];
        int a = c_tets[t][c_edges[ed][0]], b = c_tets[t][c_edges[ed][1]];
        double va = cv[a], vb = cv[b], den = vb - va;
        double tt = den != 0 ? (iso - va) / den : 0.5;
        if (tt < 0) tt = 0; else if (tt > 1) tt = 1;
        P3[vi][0] = ((i + c_corners[a][0]) + (c_corners[b][0] - c_corners[a][0]) * tt) * dx;
        P3[vi][1] = ((j + c_corners[a][1]) + (c_corners[b][1] - c_corners[a][1]) * tt) * dx;
        P3[vi][2] = ((k + c_corners[a][2]) + (c_corners[b][2] - c_corners[a][2]) * tt) * dx;
        double nxx = -(gx[a] + (gx[b] - gx[a]) * tt), nyy = -(gy[a] + (gy[b] - gy[a]) * tt), nzz = -(gz[a] + (gz[b] - gz[a]) * tt);
        double nl = sqrt(nxx * nxx + nyy * nyy + nzz * nzz); if (nl == 0) nl = 1;
        N3[vi][0] = nxx / nl; N3[vi][1] = nyy / nl; N3[vi][2] = nzz / nl;
      }
      double ux = P3[1][0] - P3[0][0], uy = P3[1][1] - P3[0][1], uz = P3[1][2] - P3[0][2];
      double vx = P3[2][0] - P3[0][0], vy = P3[2][1] - P3[0][1], vz = P3[2][2] - P3[0][2];
      double fnx = uy * vz - uz * vy, fny = uz * vx - ux * vz, fnz = ux * vy - uy * vx;
      double cgx = N3[0][0] + N3[1][0] + N3[2][0], cgy = N3[0][1] + N3[1][1] + N3[2][1], cgz = N3[0][2] + N3[1][2] + N3[2][2];
      if (fnx * cgx + fny * cgy + fnz * cgz < 0) {
        for (int q = 0; q < 3; q++) {
          double tmp = P3[2][q]; P3[2][q] = P3[1][q]; P3[1][q] = tmp;
          tmp = N3[2][q]; N3[2][q] = N3[1][q]; N3[1][q] = tmp;
        }
      }
      vol += (P3[0][0] * (P3[1][1] * P3[2][2] - P3[2][1] * P3[1][2]) -
              P3[0][1] * (P3[1][0] * P3[2][2] - P3[2][0] * P3[1][2]) +
              P3[0][2] * (P3[1][0] * P3[2][1] - P3[2][0] * P3[1][1])) / 6;
      if (pos) {
        float* pp = pos + (base + verts) * 3;
        float* nn = nrm + (base + verts) * 3;
        for (int vi = 0; vi < 3; vi++)
          for (int q = 0; q < 3; q++) { pp[vi * 3 + q] = (float)P3[vi][q]; nn[vi * 3 + q] = (float)N3[vi][q]; }
      }
      verts += 3;
    }
  }
  return vol;
}
// Cells whose corners straddle iso (the only ones mt_cell emits triangles
// for) are listed first, in index order, so the triangle work runs on full
// warps: about 2% of the cells of an ocean planet's lattice.
__global__ void k_mt_flags(Dims d, const float* __restrict__ dens, double iso, uint8_t* __restrict__ flag) {
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= d.nCells) return;
  int i, j, k; cell_ijk(d, c, i, j, k);
  const long long sj = d.nx + 1, sk = (long long)(d.ny + 1) * sj, b = k * sk + j * sj + i;
  const float v[8] = { dens[b], dens[b + 1], dens[b + sj], dens[b + sj + 1],
                       dens[b + sk], dens[b + sk + 1], dens[b + sk + sj], dens[b + sk + sj + 1] };
  double mn = v[0], mx = v[0];
#pragma unroll
  for (int q = 1; q < 8; q++) { mn = fmin(mn, (double)v[q]); mx = fmax(mx, (double)v[q]); }
  flag[c] = (mx < iso || mn > iso) ? 0 : 1;     // mt_cell's own early-out test
}
__device__ __forceinline__ int mt_chunks(const int* nList) { return (*nList + 127) >> 7; }
// Per 128-entry chunk of the list: partial sums of the signed volume (FP64)
// and the vertex count. Persistent over the chunks.
__global__ void __launch_bounds__(128, 8) k_mt_partial(Dims d, const float* __restrict__ dens, double iso,
                                                       const int* __restrict__ list, const int* __restrict__ nList,
                                                       double2* __restrict__ partials) {
  __shared__ double sv[4], sc[4];
  const int n = *nList, nch = mt_chunks(nList);
  for (int ch = blockIdx.x; ch < nch; ch += gridDim.x) {
    const int e = ch * 128 + (int)threadIdx.x;
    double vol = 0, cnt = 0;
    if (e < n) {
      int i, j, k; cell_ijk(d, list[e], i, j, k);
      int v;
      vol = mt_cell(dens, d.nx, d.ny, d.nz, d.dx, d.dxPow2 != 0, 0.5 * d.rdx, iso, i, j, k, v);
      cnt = v;
    }
    vol = warp_sum(vol); cnt = warp_sum(cnt);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { sv[wid] = vol; sc[wid] = cnt; }
    __syncthreads();
    if (threadIdx.x == 0) partials[ch] = make_double2(sv[0] + sv[1] + sv[2] + sv[3], sc[0] + sc[1] + sc[2] + sc[3]);
    __syncthreads();                              // sv, sc are rewritten by the next chunk
  }
}
// Fixed-order final reduction of double2 partials into out[0..1]; nDev (when
// given) holds a list length whose 128-entry chunks are the partials.
__global__ void k_reduce_pairs(const double2* __restrict__ partials, int n, double* __restrict__ out,
                               const int* __restrict__ nDev = nullptr) {
  __shared__ double sa[32], sb[32];
  if (nDev) n = mt_chunks(nDev);
  double a = 0, b = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) { a += partials[i].x; b += partials[i].y; }
  a = warp_sum(a); b = warp_sum(b);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { sa[wid] = a; sb[wid] = b; }
  __syncthreads();
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    a = lane < nw ? sa[lane] : 0; b = lane < nw ? sb[lane] : 0;
    a = warp_sum(a); b = warp_sum(b);
    if (lane == 0) { out[0] = a; out[1] = b; }
  }
}
size_t mt_scratch_bytes(long long nCells) {
  return (size_t)nCells + 4 * (size_t)nCells + 4 * (size_t)((nCells + 255) / 256 + 1) + 64;
}
static void mt_carve(void* scratch, long long nCells, uint8_t*& flag, int*& list, int*& blockCounts, int*& nList) {
  char* q = (char*)scratch;
  list = (int*)q; q += 4 * (size_t)nCells;
  blockCounts = (int*)q; q += 4 * (size_t)((nCells + 255) / 256 + 1);
  nList = (int*)q; q += 64;
  flag = (uint8_t*)q;
}
void launch_mt_volume(const Dims& d, const float* dens, double iso, double2* partials, double* out, void* scratch,
                      cudaStream_t s) {
  uint8_t* flag; int *list, *blockCounts, *nList;
  mt_carve(scratch, d.nCells, flag, list, blockCounts, nList);
  k_mt_flags<<<grid_for(d.nCells, 256), 256, 0, s>>>(d, dens, iso, flag);
  launch_compact(flag, (int)d.nCells, 2, blockCounts, list, nList, s);
  const int nb = (int)std::min<long long>(grid_for(d.nCells, 128), 148 * 8);
  k_mt_partial<<<nb, 128, 0, s>>>(d, dens, iso, list, nList, partials);
  k_reduce_pairs<<<1, 1024, 0, s>>>(partials, 0, out, nList);
}

// Mesh emission in the reference's order (cells in index order, then tets,
// then case triangles): exclusive scan of the per-chunk vertex counts that
// k_mt_partial left in partials[ch].y, then each chunk of the straddling-cell
// list places its cells' vertices by a block scan of their counts.
__global__ void k_mt_offsets(const double2* __restrict__ partials, const int* __restrict__ nList, long long* __restrict__ offs) {
  __shared__ long long ws[32], carry;
  const int nb = mt_chunks(nList);
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int base = 0; base < nb; base += blockDim.x) {
    int i = base + threadIdx.x;
    long long v = i < nb ? llround(partials[i].y) : 0, x = v;
    for (int o = 1; o < 32; o <<= 1) { long long y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    if (w == 0) {
      long long a = lane < nw ? ws[lane] : 0;
      for (int o = 1; o < 32; o <<= 1) { long long y = __shfl_up_sync(0xffffffffu, a, o); if (lane >= o) a += y; }
      ws[lane] = a;
    }
    __syncthreads();
    long long ex = x - v + (w > 0 ? ws[w - 1] : 0) + carry;
    if (i < nb) offs[i] = ex;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = ex + v;
    __syncthreads();
  }
}
__global__ void __launch_bounds__(128, 8) k_mt_emit(Dims d, const float* __restrict__ dens, double iso,
                                                    const int* __restrict__ list, const int* __restrict__ nList,
                                                    const long long* __restrict__ offs, long long maxVerts,
                                                    float* __restrict__ pos, float* __restrict__ nrm) {
  __shared__ int ws[4];
  const int n = *nList, nch = mt_chunks(nList);
  for (int ch = blockIdx.x; ch < nch; ch += gridDim.x) {
    const int e = ch * 128 + (int)threadIdx.x;
    int i = 0, j = 0, k = 0, v = 0;
    if (e < n) {
      cell_ijk(d, list[e], i, j, k);
      mt_cell(dens, d.nx, d.ny, d.nz, d.dx, d.dxPow2 != 0, 0.5 * d.rdx, iso, i, j, k, v);
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) { int y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    int before = 0;
    for (int q = 0; q < w; q++) before += ws[q];
    const long long base = offs[ch] + before + x - v;
    if (v > 0 && base + v <= maxVerts) {
      int v2;
      mt_cell(dens, d.nx, d.ny, d.nz, d.dx, d.dxPow2 != 0, 0.5 * d.rdx, iso, i, j, k, v2, pos, nrm, base);
    }
    __syncthreads();                              // ws is rewritten by the next chunk
  }
}
void launch_mt_mesh(const Dims& d, const float* dens, double iso, const double2* partials, long long* offs,
                    long long maxVerts, float* pos, float* nrm, void* scratch, cudaStream_t s) {
  uint8_t* flag; int *list, *blockCounts, *nList;
  mt_carve(scratch, d.nCells, flag, list, blockCounts, nList);
  const int nb = (int)std::min<long long>(grid_for(d.nCells, 128), 148 * 8);
  k_mt_offsets<<<1, 1024, 0, s>>>(partials, nList, offs);
  k_mt_emit<<<nb, 128, 0, s>>>(d, dens, iso, list, nList, offs, maxVerts, pos, nrm);
}

// ------------------------------------------------------------ particle reductions
// mode 0: kinetic energy sum of 0.5 mp v^2 (FP64); mode 1: census counts
// (liquid 0/1/4, ice 5, vapour 2/3) as exact FP64 integers.
__global__ void k_particle_reduce(PartsDev P, int mode, double mp, double* __restrict__ partials) {
  __shared__ double s0[32], s1[32], s2[32];
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  double a = 0, b = 0, c = 0;
  if (p < P.nP) {
    if (mode == 0) {
      double vx = P.pvx[p], vy = P.pvy[p], vz = P.pvz[p];
      a = 0.5 * mp * (vx * vx + vy * vy + vz * vz);
    } else {
      int f = P.pflag[p];
      if (f == 0 || f == 1 || f == 4) a = 1; else if (f == 5) b = 1; else if (f == 2 || f == 3) c = 1;
    }
  }
  a = warp_sum(a); b = warp_sum(b); c = warp_sum(c);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { s0[wid] = a; s1[wid] = b; s2[wid] = c; }
  __syncthreads();
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    a = lane < nw ? s0[lane] : 0; b = lane < nw ? s1[lane] : 0; c = lane < nw ? s2[lane] : 0;
    a = warp_sum(a); b = warp_sum(b); c = warp_sum(c);
    if (lane == 0) { partials[3 * blockIdx.x] = a; partials[3 * blockIdx.x + 1] = b; partials[3 * blockIdx.x + 2] = c; }
  }
}
__global__ void k_reduce_triples(const double* __restrict__ partials, int n, double* __restrict__ out) {
  if (threadIdx.x == 0) {
    double a = 0, b = 0, c = 0;
    for (int i = 0; i < n; i++) { a += partials[3 * i]; b += partials[3 * i + 1]; c += partials[3 * i + 2]; }
    out[0] = a; out[1] = b; out[2] = c;
  }
}
void launch_particle_reduce(const PartsDev& P, int mode, double mp, double* partials, double* out, cudaStream_t s) {
  int nb = (int)grid_for(P.nP > 0 ? P.nP : 1, 256);
  k_particle_reduce<<<nb, 256, 0, s>>>(P, mode, mp, partials);
  k_reduce_triples<<<1, 32, 0, s>>>(partials, nb, out);
}

// ------------------------------------------------------------ subsurface currents
// js/solver.js:3624-3782. The curl of a drifting sum-of-sines vector
// potential on a lattice of stride 4 cells (float storage), then a capped
// relaxation of deep fluid particles toward its tangential part. The nine
// waves come from the reference's fixed seeded LCG (host, CurrWaves).
__global__ void k_curr_field(CurrField F, double t, double ampl) {
  long long gi = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long gN = (long long)F.gnx * F.gny * F.gnz;
  if (gi >= gN) return;
  const int ii = (int)(gi % F.gnx), jj = (int)((gi / F.gnx) % F.gny), kk = (int)(gi / ((long long)F.gnx * F.gny));
  const double wx2 = ii * F.sx, wy2 = jj * F.sx, wz2 = kk * F.sx;
  double ux = 0, uy = 0, uz = 0;
  for (int o = 0; o < 3; o++) {
    const double* w0 = F.w + (o * 3 + 0) * 5;
    const double* w1 = F.w + (o * 3 + 1) * 5;
    const double* w2 = F.w + (o * 3 + 2) * 5;
    const double dph = F.drift[o] * t;
    const double thx = w0[0] * wx2 + w0[1] * wy2 + w0[2] * wz2 + dph + w0[4];
    const double thy = w1[0] * wx2 + w1[1] * wy2 + w1[2] * wz2 + dph + w1[4];
    const double thz = w2[0] * wx2 + w2[1] * wy2 + w2[2] * wz2 + dph + w2[4];
    ux += w2[3] * w2[1] * cos(thz) - w1[3] * w1[2] * cos(thy);
    uy += w0[3] * w0[2] * cos(thx) - w2[3] * w2[0] * cos(thz);
    uz += w1[3] * w1[0] * cos(thy) - w0[3] * w0[1] * cos(thx);
  }
  F.cfx[gi] = (float)(ux * ampl); F.cfy[gi] = (float)(uy * ampl); F.cfz[gi] = (float)(uz * ampl);
}
__global__ void k_currents(Dims d, PartsDev P, CurrField F, double oceanR, double shell, double relax, int kmax) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nP || P.pflag[p] != 0) return;
  const double dvCap = 0.15, invS = 1 / F.sx;
  double rx = P.px[p] - d.cx, ry = P.py[p] - d.cy, rz = P.pz[p] - d.cz;
  double rl = sqrt(rx * rx + ry * ry + rz * rz); if (rl == 0) rl = 1e-9;
  const double dpt = (oceanR - rl) / shell;
  double wgt = (dpt - 0.06) * 4.0;
  if (wgt <= 0) return;
  if (wgt > 1) wgt = 1;
  const double qa = P.px[p] * invS, qb = P.py[p] * invS, qc = P.pz[p] * invS;
  int i0 = jtrunc(qa), j0 = jtrunc(qb), k0 = jtrunc(qc);
  if (i0 > F.gnx - 2) i0 = F.gnx - 2; else if (i0 < 0) i0 = 0;
  if (j0 > F.gny - 2) j0 = F.gny - 2; else if (j0 < 0) j0 = 0;
  if (k0 > kmax) k0 = kmax; else if (k0 < 0) k0 = 0;
  double ta = qa - i0; if (ta > 1) ta = 1; else if (ta < 0) ta = 0;
  double tb = qb - j0; if (tb > 1) tb = 1; else if (tb < 0) tb = 0;
  double tc = qc - k0; if (tc > 1) tc = 1; else if (tc < 0) tc = 0;
  const long long gnx = F.gnx, gxy = (long long)F.gnx * F.gny, g = (k0 * (long long)F.gny + j0) * gnx + i0;
  const double a0 = 1 - ta, a1 = ta, b0 = 1 - tb, b1 = tb, c0 = 1 - tc, c1 = tc;
  auto samp = [&](const float* f) -> double {
    return ((double)f[g] * a0 + (double)f[g + 1] * a1) * b0 * c0 + ((double)f[g + gnx] * a0 + (double)f[g + gnx + 1] * a1) * b1 * c0 +
           ((double)f[g + gxy] * a0 + (double)f[g + gxy + 1] * a1) * b0 * c1 +
           ((double)f[g + gxy + gnx] * a0 + (double)f[g + gxy + gnx + 1] * a1) * b1 * c1;
  };
  const double Ux = samp(F.cfx), Uy = samp(F.cfy), Uz = samp(F.cfz);
  const double ir = 1 / rl;
  const double Ur = (Ux * rx + Uy * ry + Uz * rz) * ir;
  const double Tx = (Ux - rx * ir * Ur) * wgt, Ty = (Uy - ry * ir * Ur) * wgt, Tz = (Uz - rz * ir * Ur) * wgt;
  const double vr = ((double)P.pvx[p] * rx + (double)P.pvy[p] * ry + (double)P.pvz[p] * rz) * ir;
  const double vx = P.pvx[p] - rx * ir * vr, vy = P.pvy[p] - ry * ir * vr, vz = P.pvz[p] - rz * ir * vr;
  double ex = relax * (Tx - vx), ey = relax * (Ty - vy), ez = relax * (Tz - vz);
  const double e2 = ex * ex + ey * ey + ez * ez;
  if (e2 > dvCap * dvCap) { const double es = dvCap / sqrt(e2); ex *= es; ey *= es; ez *= es; }
  P.pvx[p] = (float)(P.pvx[p] + ex); P.pvy[p] = (float)(P.pvy[p] + ey); P.pvz[p] = (float)(P.pvz[p] + ez);
}
void launch_currents(const Dims& d, const PartsDev& P, const CurrField& F, double simTime, double strength,
                     double oceanR, double coreR, double dt, cudaStream_t s) {
  const double shell = oceanR - coreR;
  if (!(strength > 0) || !(shell > 0)) return;
  const long long gN = (long long)F.gnx * F.gny * F.gnz;
  k_curr_field<<<grid_for(gN, 256), 256, 0, s>>>(F, simTime, strength * 2);
  double relax = 2.2 * dt; if (relax > 0.35) relax = 0.35;
  if (P.nP > 0) k_currents<<<grid_for(P.nP, 256), 256, 0, s>>>(d, P, F, oceanR, shell, relax, d.nz / 4);
}

// ---------------------------------------------------------------- metaballs
// Metaballs.build's kernel field (js/surface.js:248-283): every liquid
// particle adds (1 - d^2/R^2)^2 to the corners of the (m+1)^3 lattice within
// R (stencil +-rad around the rounded lattice position, clamped to the
// lattice). The reference sums in Float32 in particle order; here each corner
// accumulates in FP64 (any order) and is rounded to float once, so the field
// is deterministic and within the reference's own float rounding of it.
__device__ __forceinline__ double js_round(double x) { double r = floor(x); return (x - r >= 0.5) ? r + 1 : r; }
__global__ void k_mb_splat(PartsDev P, int m, double mdx, double R2, int rad, double* __restrict__ acc) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nP || P.pflag[p] != 0) return;
  const double gx = P.px[p] / mdx, gy = P.py[p] / mdx, gz = P.pz[p] / mdx;
  // outside (-8, m + 8) (or NaN) the reference's clamped ranges are empty
  if (!(gx > -8 && gx < m + 8 && gy > -8 && gy < m + 8 && gz > -8 && gz < m + 8)) return;
  const int i0 = (int)js_round(gx), j0 = (int)js_round(gy), k0 = (int)js_round(gz);
  const int ia = max(i0 - rad, 0), ib = min(i0 + rad, m);
  const int ja = max(j0 - rad, 0), jb = min(j0 + rad, m);
  const int ka = max(k0 - rad, 0), kb = min(k0 + rad, m);
  const long long sj = m + 1, sk = (long long)(m + 1) * sj;
  for (int k = ka; k <= kb; k++) {
    const double ez = k - gz, dz2 = ez * ez;
    if (dz2 >= R2) continue;
    for (int j = ja; j <= jb; j++) {
      const double ey = j - gy, dy2 = dz2 + ey * ey;
      if (dy2 >= R2) continue;
      const long long base = k * sk + j * sj;
      for (int i = ia; i <= ib; i++) {
        const double ex = i - gx, d2 = dy2 + ex * ex;
        if (d2 >= R2) continue;
        const double u = 1 - d2 / R2;
        atomicAdd(acc + base + i, u * u);
      }
    }
  }
}
__global__ void k_mb_round(const double* __restrict__ acc, float* __restrict__ field, long long n) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
    field[c] = (float)acc[c];
}
void launch_metaball_field(const PartsDev& P, int m, double mdx, double R2, int rad, double* acc, float* field,
                           cudaStream_t s) {
  const long long corners = (long long)(m + 1) * (m + 1) * (m + 1);
  cudaMemsetAsync(acc, 0, sizeof(double) * (size_t)corners, s);
  if (P.nP) k_mb_splat<<<grid_for(P.nP, 256), 256, 0, s>>>(P, m, mdx, R2, rad, acc);
  k_mb_round<<<(int)std::min<long long>(grid_for(corners, 256), 148 * 16), 256, 0, s>>>(acc, field, corners);
}
