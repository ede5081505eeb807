// ws_contacts.cu — frame-level contact passes: _vaporCollisions
// (js/solver.js:3345-3479) and _iceContacts (:3290-3324).
//
// The reference resolves pairs in place, one after another in sorted-x
// order, so each pair sees the updates of the pairs before it.
// - Vapour contacts: the device resolves every pair from one snapshot of the
//   state (Jacobi order) and sums the equal-and-opposite impulses with
//   atomics. Pair momentum is conserved exactly as in the reference; the
//   per-particle result differs at second order where one parcel touches
//   several others in the same frame. The vapour census (vaporCount,
//   nightVaporCount) is exact.
// - Ice contacts: exact. The sorted list is cut where neighbours are at
//   least the contact radius apart in x; no pair crosses such a gap, so each
//   segment is swept serially by one thread in the reference's order.
// The x-sort uses CUB's device radix sort (a CUDA toolkit library).
#include "ws_kernels.cuh"
#include <cub/cub.cuh>

struct ContactScratch {
  int *idxA, *idxB, *blockCounts, *nV;
  uint32_t *keyA, *keyB;
  float *snap, *acc;       // 6 floats per contact particle (x, y, z, vx, vy, vz)
  int *perm, *rowStart;    // parcels by grid row (j, k): snapshot index, first parcel of each row
  void* cubTemp;
  size_t cubBytes;
};

static size_t cub_bytes(int cap) {
  size_t bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, bytes, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                  (int*)nullptr, (int*)nullptr, cap);
  return bytes;
}
static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
size_t contacts_scratch_bytes(int cap, int rows) {
  size_t nb = (size_t)(cap + 255) / 256 + 1;
  return align256(4 * (size_t)cap) * 5 + align256(4 * nb) + 256 + align256(24 * (size_t)cap) * 2 +
         align256(4 * ((size_t)rows + 1)) + align256(cub_bytes(cap));
}
static ContactScratch carve(void* base, int cap, int rows) {
  char* p = (char*)base; ContactScratch c;
  size_t nb = (size_t)(cap + 255) / 256 + 1;
  c.idxA = (int*)p; p += align256(4 * (size_t)cap);
  c.idxB = (int*)p; p += align256(4 * (size_t)cap);
  c.keyA = (uint32_t*)p; p += align256(4 * (size_t)cap);
  c.keyB = (uint32_t*)p; p += align256(4 * (size_t)cap);
  c.blockCounts = (int*)p; p += align256(4 * nb);
  c.nV = (int*)p; p += 256;
  c.snap = (float*)p; p += align256(24 * (size_t)cap);
  c.acc = (float*)p; p += align256(24 * (size_t)cap);
  c.perm = (int*)p; p += align256(4 * (size_t)cap);
  c.rowStart = (int*)p; p += align256(4 * ((size_t)rows + 1));
  c.cubTemp = p; c.cubBytes = cub_bytes(cap);
  return c;
}

// exact vapour census (:3350-3360)
__global__ void k_vapor_census(Dims d, PartsDev P, int hasSun, double sx, double sy, double sz, DevStatus* st) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  int steam = 0, night = 0;
  if (p < P.nP && P.pflag[p] == 2) {
    steam = 1;
    if (!hasSun || ((double)P.px[p] - d.cx) * sx + ((double)P.py[p] - d.cy) * sy + ((double)P.pz[p] - d.cz) * sz < 0) night = 1;
  }
  steam = warp_sum(steam); night = warp_sum(night);
  if ((threadIdx.x & 31) == 0) { if (steam) atomicAdd(&st->vaporCount, steam); if (night) atomicAdd(&st->nightVapor, night); }
}
__global__ void k_keys(const int* __restrict__ idx, const int* __restrict__ nV, const float* __restrict__ px, uint32_t* __restrict__ key) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= *nV) return;
  key[i] = __float_as_uint(px[idx[i]]);      // positions are positive: bit order == value order
}
__global__ void k_snapshot(PartsDev P, const int* __restrict__ idx, int n, float* __restrict__ snap, float* __restrict__ acc) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int p = idx[i];
  snap[6 * i] = P.px[p]; snap[6 * i + 1] = P.py[p]; snap[6 * i + 2] = P.pz[p];
  snap[6 * i + 3] = P.pvx[p]; snap[6 * i + 4] = P.pvy[p]; snap[6 * i + 5] = P.pvz[p];
  for (int q = 0; q < 6; q++) acc[6 * i + q] = 0.f;
}
// vapour-vapour pairs (:3371-3396): elastic normal exchange when
// approaching, positional separation and a soft repulsion kick always
__global__ void k_vv_pairs(const float* __restrict__ snap, int n, double rad, float* __restrict__ acc) {
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  const float* A = snap + 6 * a;
  double rad2 = rad * rad;
  for (int b = a + 1; b < n; b++) {
    const float* B = snap + 6 * b;
    double ddx = (double)B[0] - A[0];
    if (ddx >= rad) break;
    double ddy = (double)B[1] - A[1], ddz = (double)B[2] - A[2];
    double d2 = ddx * ddx + ddy * ddy + ddz * ddz;
    if (d2 >= rad2) continue;
    double dd = sqrt(d2); if (dd == 0) dd = 1e-9;
    double nX = ddx / dd, nY = ddy / dd, nZ = ddz / dd;
    double vRel = ((double)A[3] - B[3]) * nX + ((double)A[4] - B[4]) * nY + ((double)A[5] - B[5]) * nZ;
    double dv = (vRel > 0 ? vRel : 0) + (rad - dd) * 2;
    double half = (rad - dd) * 0.5;
    atomicAdd(&acc[6 * a + 0], (float)(-nX * half)); atomicAdd(&acc[6 * a + 1], (float)(-nY * half)); atomicAdd(&acc[6 * a + 2], (float)(-nZ * half));
    atomicAdd(&acc[6 * b + 0], (float)(nX * half)); atomicAdd(&acc[6 * b + 1], (float)(nY * half)); atomicAdd(&acc[6 * b + 2], (float)(nZ * half));
    atomicAdd(&acc[6 * a + 3], (float)(-nX * dv)); atomicAdd(&acc[6 * a + 4], (float)(-nY * dv)); atomicAdd(&acc[6 * a + 5], (float)(-nZ * dv));
    atomicAdd(&acc[6 * b + 3], (float)(nX * dv)); atomicAdd(&acc[6 * b + 4], (float)(nY * dv)); atomicAdd(&acc[6 * b + 5], (float)(nZ * dv));
  }
}
// Grid rows (j, k) of the snapshot's parcels. The snapshot is in x order and
// the row sort is stable, so each row's parcels stay in x order.
__global__ void k_row_keys(Dims d, const float* __restrict__ snap, int n, uint32_t* __restrict__ key,
                           int* __restrict__ val) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int j = jtrunc(over_dx(d, snap[6 * i + 1])), k = jtrunc(over_dx(d, snap[6 * i + 2]));
  j = j < 0 ? 0 : (j >= d.ny ? d.ny - 1 : j);
  k = k < 0 ? 0 : (k >= d.nz ? d.nz - 1 : k);
  key[i] = (uint32_t)(k * d.ny + j);
  val[i] = i;
}
// rowStart[r] = first sorted parcel with row >= r, for r = 0 .. rows (rowStart[rows] = n)
__global__ void k_row_starts(const uint32_t* __restrict__ key, int n, int rows, int* __restrict__ rowStart) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r > rows) return;
  int lo = 0, hi = n;
  while (lo < hi) { int mid = (lo + hi) >> 1; if (key[mid] < (uint32_t)r) lo = mid + 1; else hi = mid; }
  rowStart[r] = lo;
}
// liquid-vapour contacts (:3433-3478): only the parcel moves. The reference
// tests every parcel of the x-sorted list within rad in x; the device tests
// the same condition on the parcels of the grid rows that rad reaches in y
// and z (a parcel outside them is farther than rad), so the contact set is
// the same.
__global__ void k_vl_pairs(Dims d, PartsDev P, const float* __restrict__ snap, const int* __restrict__ perm,
                           const int* __restrict__ rowStart, double rad, double bandLo2, float* __restrict__ acc) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nP) return;
  int fw = P.pflag[p];
  if (fw != 0 && fw != 1 && fw != 4) return;
  double wx = P.px[p], wy = P.py[p], wz = P.pz[p];
  if (fw == 0) {
    double ex = wx - d.cx, ey = wy - d.cy, ez = wz - d.cz;
    if (ex * ex + ey * ey + ez * ez < bandLo2) return;
  }
  const double radq = rad + 1e-6 * d.dx;         // rows reached, widened past rounding
  int j0 = jfloor_clamp(over_dx(d, wy - radq), 0, d.ny - 1), j1 = jfloor_clamp(over_dx(d, wy + radq), 0, d.ny - 1);
  int k0 = jfloor_clamp(over_dx(d, wz - radq), 0, d.nz - 1), k1 = jfloor_clamp(over_dx(d, wz + radq), 0, d.nz - 1);
  double wvx = P.pvx[p], wvy = P.pvy[p], wvz = P.pvz[p], rad2 = rad * rad;
  for (int k = k0; k <= k1; k++) {
    for (int j = j0; j <= j1; j++) {
      const int r = k * d.ny + j;
      const int m1 = rowStart[r + 1];
      for (int m = rowStart[r]; m < m1; m++) {
        const int b = perm[m];
        const float* B = snap + 6 * b;
        if ((double)B[0] < wx - rad) continue;
        double ddx = (double)B[0] - wx;
        if (ddx >= rad) break;                     // the row is in x order
        double ddy = (double)B[1] - wy, ddz = (double)B[2] - wz;
        double dd2 = ddx * ddx + ddy * ddy + ddz * ddz;
        if (dd2 >= rad2 || dd2 < 1e-12) continue;
        double dd = sqrt(dd2), nX = ddx / dd, nY = ddy / dd, nZ = ddz / dd;
        double vR = ((double)B[3] - wvx) * nX + ((double)B[4] - wvy) * nY + ((double)B[5] - wvz) * nZ;
        double ov = rad - dd, dv = ov * 2 - (vR < 0 ? vR * 1.4 : 0);
        atomicAdd(&acc[6 * b + 0], (float)(nX * ov)); atomicAdd(&acc[6 * b + 1], (float)(nY * ov)); atomicAdd(&acc[6 * b + 2], (float)(nZ * ov));
        atomicAdd(&acc[6 * b + 3], (float)(nX * dv)); atomicAdd(&acc[6 * b + 4], (float)(nY * dv)); atomicAdd(&acc[6 * b + 5], (float)(nZ * dv));
      }
    }
  }
}
__global__ void k_apply(PartsDev P, const int* __restrict__ idx, int n, const float* __restrict__ acc) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int p = idx[i];
  P.px[p] = (float)((double)P.px[p] + acc[6 * i]); P.py[p] = (float)((double)P.py[p] + acc[6 * i + 1]);
  P.pz[p] = (float)((double)P.pz[p] + acc[6 * i + 2]);
  P.pvx[p] = (float)((double)P.pvx[p] + acc[6 * i + 3]); P.pvy[p] = (float)((double)P.pvy[p] + acc[6 * i + 4]);
  P.pvz[p] = (float)((double)P.pvz[p] + acc[6 * i + 5]);
}

static int sorted_list(const PartsDev& P, int mode, ContactScratch& c, int* hostN, cudaStream_t s) {
  launch_compact(P.pflag, P.nP, mode, c.blockCounts, c.idxA, c.nV, s);
  cudaMemcpyAsync(hostN, c.nV, sizeof(int), cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  int n = *hostN;
  if (n < 2) return n;
  k_keys<<<grid_for(n, 256), 256, 0, s>>>(c.idxA, c.nV, P.px, c.keyA);
  size_t bytes = c.cubBytes;
  cub::DeviceRadixSort::SortPairs(c.cubTemp, bytes, c.keyA, c.keyB, c.idxA, c.idxB, n, 0, 32, s);
  return n;
}

void launch_vapor_collisions(const Dims& d, const PartsDev& P, double spacing, double oceanR, int spinOn,
                             int hasSun, const double* sunRel, void* scratch, size_t scratchBytes,
                             DevStatus* st, cudaStream_t s) {
  (void)spinOn; (void)scratchBytes;
  cudaMemsetAsync(&st->vaporCount, 0, 2 * sizeof(int), s);
  if (P.nP <= 0) return;
  k_vapor_census<<<grid_for(P.nP, 256), 256, 0, s>>>(d, P, hasSun, sunRel[0], sunRel[1], sunRel[2], st);
  const int rows = d.ny * d.nz;
  ContactScratch c = carve(scratch, P.nP > 0 ? P.nP : 1, rows);
  int hostN = 0;
  int n = sorted_list(P, 0, c, &hostN, s);
  if (n < 2) return;
  double rad = spacing * 0.6;
  k_snapshot<<<grid_for(n, 256), 256, 0, s>>>(P, c.idxB, n, c.snap, c.acc);
  k_vv_pairs<<<grid_for(n, 128), 128, 0, s>>>(c.snap, n, rad, c.acc);
  int rowBits = 1;
  while ((1ll << rowBits) < (long long)rows) rowBits++;
  k_row_keys<<<grid_for(n, 256), 256, 0, s>>>(d, c.snap, n, c.keyA, c.idxA);
  size_t bytes = c.cubBytes;
  cub::DeviceRadixSort::SortPairs(c.cubTemp, bytes, c.keyA, c.keyB, c.idxA, c.perm, n, 0, rowBits, s);
  k_row_starts<<<grid_for(rows + 1, 256), 256, 0, s>>>(c.keyB, n, rows, c.rowStart);
  double band = oceanR - d.dx * 2;
  k_vl_pairs<<<grid_for(P.nP, 256), 256, 0, s>>>(d, P, c.snap, c.perm, c.rowStart, rad, band * band, c.acc);
  k_apply<<<grid_for(n, 256), 256, 0, s>>>(P, c.idxB, n, c.acc);
}

// _iceContacts (:3290-3324), exact. The reference sweeps the x-sorted ice
// list serially: pair (a, b) sees every update of the pairs before it. The
// sweep of grain a only reaches grains b with px[b] - px[a] < rad, so a gap of
// at least rad between neighbours in the sorted list cuts it into segments
// no pair crosses. Each segment is swept by one thread in the reference's
// order, with the reference's arithmetic, on the live particle arrays; the
// segments touch disjoint particles, so their sweeps run in parallel and the
// result is the serial sweep's, bit for bit.
__global__ void k_ice_segments(const float* __restrict__ px, const int* __restrict__ idx, int n, double rad,
                               uint8_t* __restrict__ segStart) {
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  segStart[a] = a == 0 || (double)px[idx[a]] - (double)px[idx[a - 1]] >= rad;
}
__global__ void k_ice_sweep(PartsDev P, const int* __restrict__ idx, const uint8_t* __restrict__ segStart, int n,
                            double rad) {
  int s0 = blockIdx.x * blockDim.x + threadIdx.x;
  if (s0 >= n || !segStart[s0]) return;
  const double rad2 = rad * rad;
  const float *px = P.px, *py = P.py, *pz = P.pz;
  float *pvx = P.pvx, *pvy = P.pvy, *pvz = P.pvz, *pAir = P.pAir;
  for (int a = s0; a < n && (a == s0 || !segStart[a]); a++) {
    const int i = idx[a];
    bool stuckI = pAir[i] == 1.f;
    for (int b = a + 1; b < n; b++) {
      const int j = idx[b];
      if ((double)px[j] - (double)px[i] >= rad) break;
      double ddx = (double)px[j] - (double)px[i], ddy = (double)py[j] - (double)py[i], ddz = (double)pz[j] - (double)pz[i];
      if (ddx * ddx + ddy * ddy + ddz * ddz >= rad2) continue;
      const bool stuckJ = pAir[j] == 1.f;
      if (stuckI && stuckJ) continue;
      if (stuckJ) {                    // free i lands on the pack at j
        pAir[i] = 1.f; pvx[i] = pvy[i] = pvz[i] = 0.f; stuckI = true;
      } else if (stuckI) {             // free j lands on the pack at i
        pAir[j] = 1.f; pvx[j] = pvy[j] = pvz[j] = 0.f;
      } else {                         // two free grains: both take the mean velocity
        const float mx = (float)(((double)pvx[i] + (double)pvx[j]) * 0.5);
        const float my = (float)(((double)pvy[i] + (double)pvy[j]) * 0.5);
        const float mz = (float)(((double)pvz[i] + (double)pvz[j]) * 0.5);
        pvx[i] = pvx[j] = mx; pvy[i] = pvy[j] = my; pvz[i] = pvz[j] = mz;
      }
    }
  }
}
__global__ void k_ice_flags(const uint8_t* __restrict__ fl, int nP, uint8_t* __restrict__ out) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < nP) out[p] = fl[p] == 5;
}
void launch_ice_contacts(const PartsDev& P, double spacing, void* scratch, size_t scratchBytes, cudaStream_t s) {
  (void)scratchBytes;
  if (P.nP <= 1) return;
  ContactScratch c = carve(scratch, P.nP, 1);
  // ice list: compact pflag == 5 via a byte predicate in the snapshot buffer
  uint8_t* pred = (uint8_t*)c.acc;
  k_ice_flags<<<grid_for(P.nP, 256), 256, 0, s>>>(P.pflag, P.nP, pred);
  launch_compact(pred, P.nP, 2, c.blockCounts, c.idxA, c.nV, s);
  int hostN = 0;
  cudaMemcpyAsync(&hostN, c.nV, sizeof(int), cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  int n = hostN;
  if (n < 2) return;
  k_keys<<<grid_for(n, 256), 256, 0, s>>>(c.idxA, c.nV, P.px, c.keyA);
  size_t bytes = c.cubBytes;
  cub::DeviceRadixSort::SortPairs(c.cubTemp, bytes, c.keyA, c.keyB, c.idxA, c.idxB, n, 0, 32, s);
  uint8_t* segStart = (uint8_t*)c.acc;
  k_ice_segments<<<grid_for(n, 256), 256, 0, s>>>(P.px, c.idxB, n, spacing * 0.7, segStart);
  k_ice_sweep<<<grid_for(n, 128), 128, 0, s>>>(P, c.idxB, segStart, n, spacing * 0.7);
}
