// ws_render.cu — render-side particle prep on the device.
//
// WaterScene.updateParticles (js/scene.js:1595-1922) stages every particle
// into one of five draw classes (liquid beads, spray/rain, vapour, cloud,
// snow), colours it (sun exposure, temperature tint, spin twinkle, or the
// spin-velocity palette), then counting-sorts the concatenation of the
// classes far-to-near into 64 buckets of squared camera distance and writes
// the sorted draw list (position, colour, alpha, size, sprite tile).
//
// The ordering the reference produces is: bucket descending, then class in
// the order above, then particle index. That is a stable counting sort of the
// particle array itself on the composite key (63 - bucket) * 5 + class — no
// per-class staging is needed. Four launches:
//   k_rp_classify  class + squared distance per particle, class counts,
//                  min/max of the drawn distances and of the spin components
//   k_rp_hist      per-chunk histogram of the 320 keys
//   k_rp_scan      exclusive scan of each key's chunk counts, key totals
//   k_rp_emit      stable rank inside the chunk (warp match + per-warp
//                  running counters), colour, draw-list write
// Double arithmetic, float stores, no contraction (built with -fmad=false):
// positions, ordering, alpha, size and sprite match the reference bit for
// bit; colours (Math.pow as exp(1.4 log t), Math.cos as cos) agree with the
// reference to the last float ulp.
#include "ws_internal.cuh"
#include "ws_kernels.cuh"
#include <algorithm>

namespace {

constexpr int kThreads = 256, kWarps = 8, kRounds = 8;
constexpr int kChunk = kWarps * kRounds * 32;      // particles per block, 256 per warp
constexpr int kKeys = 64 * 5;
constexpr unsigned char kCulled = 255;
constexpr unsigned char kSunny = 8;                  // class byte: day-side liquid bead

// reduction words: 0-4 class counts, 5-7 spin max (ordered), 8 d2 max bits,
// 9 d2 min bits, 10-12 spin min (ordered)
enum { R_CNT = 0, R_WMAX = 5, R_DMAX = 8, R_DMIN = 9, R_WMIN = 10, R_WORDS = 13 };

__device__ __forceinline__ unsigned ord_of(float f) {
  unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ double float_of(unsigned k) {
  return (double)__uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

struct Spin { double m[3], r[3]; };

__device__ __forceinline__ Spin spin_scale(const unsigned* red) {
  Spin s;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    double lo = float_of(red[R_WMIN + d]), hi = float_of(red[R_WMAX + d]);
    s.m[d] = lo;
    s.r[d] = hi > lo ? 1 / (hi - lo) : 0;
  }
  return s;
}

// bucket origin and scale: js/scene.js:1851-1858; no sort → one bucket
__device__ __forceinline__ void bucket_scale(const RenderCfg& c, const unsigned* red, double* lo, double* inv) {
  unsigned total = red[0] + red[1] + red[2] + red[3] + red[4];
  *lo = 0; *inv = 0;
  if (!c.sortOn || total <= 1) return;
  double l = (double)__uint_as_float(red[R_DMIN]), h = (double)__uint_as_float(red[R_DMAX]);
  *lo = l;
  *inv = h > l ? 63 / (h - l + 1e-9) : 0;
}
__device__ __forceinline__ int key_of(int cls, float d2, double lo, double inv) {
  int bk = (int)(((double)d2 - lo) * inv);
  bk = bk < 0 ? 0 : (bk > 63 ? 63 : bk);
  return (63 - bk) * 5 + cls;
}

__device__ __forceinline__ float dist2(const RenderCfg& c, float x, float y, float z) {
  double dx = x - c.cam[0], dy = y - c.cam[1], dz = z - c.cam[2];
  return (float)(dx * dx + dy * dy + dz * dz);
}

// js/scene.js:1720-1744: draw class of one particle (or -1 when it is not
// drawn); sunnyBead marks a liquid bead on the day side (kept with the class
// byte for the colour pass). The depth byte is read only for a night-side bead.
__device__ __forceinline__ int rp_class(const RenderCfg& c, int f, float x, float y, float z, const uint8_t* depth,
                                        bool* sunnyBead) {
  *sunnyBead = false;
  if (f == 3) return c.showSpray ? 3 : -1;
  if (f == 5) return c.showSpray ? 4 : -1;
  if (f == 2) return c.showSpray ? 2 : -1;
  if (f != 0) return c.showSpray ? 1 : -1;
  if (!c.showBeads) return -1;
  bool sunny = !c.planetLit;
  if (!sunny) {
    double sx = x - c.center[0], sy = y - c.center[1], sz = z - c.center[2];
    double sl = sqrt(sx * sx + sy * sy + sz * sz);
    if (!(sl > 0)) sl = 1e-6;
    sunny = (sx * c.sun[0] + sy * c.sun[1] + sz * c.sun[2]) / (sl * 1) > 0;
  }
  if (!sunny && depth && c.useDepth && __ldg(depth) > 1) return -1;
  *sunnyBead = sunny;
  return 0;
}

// js/scene.js:1659-1690, 1701-1774: the colour of a drawn particle as the
// reference's Float32Array staging holds it
__device__ __forceinline__ void rp_color(const RenderCfg& c, const PartsDev& P, int p, int cls, int f, bool sunnyBead,
                                         float x, float y, float z, const Spin& sp, float* col) {
  if (c.spinCol) {
    col[0] = (float)(sp.r[0] ? (__ldg(P.pWx + p) - sp.m[0]) * sp.r[0] : 0.5);
    col[1] = (float)(sp.r[1] ? (__ldg(P.pWy + p) - sp.m[1]) * sp.r[1] : 0.5);
    col[2] = (float)(sp.r[2] ? (__ldg(P.pWz + p) - sp.m[2]) * sp.r[2] : 0.5);
    return;
  }
  double expo = 1;
  if (c.planetLit) {
    if (c.useLight) {
      expo = __ldg(P.pLight + p);
      if (!(expo > 0)) expo = 0; else if (expo > 1) expo = 1;
    } else {
      double ex = x - c.center[0], ey = y - c.center[1], ez = z - c.center[2];
      double el = sqrt(ex * ex + ey * ey + ez * ez);
      if (!(el > 0)) el = 1e-6;
      expo = (ex * c.sun[0] + ey * c.sun[1] + ez * c.sun[2]) / (el * 1);
      if (expo < 0) expo = 0;
    }
  }
  const double br = 0.12 + 0.88 * expo;
  if (cls == 3) {
    double cl = 0.30 + 0.70 * br;
    if (c.spinCue) cl *= 0.9 + 0.1 * cos((double)__ldg(P.pPh + p));
    col[0] = (float)(0.88 * cl); col[1] = (float)(0.90 * cl); col[2] = (float)(0.93 * cl);
  } else if (cls == 4) {
    double sw = 0.62 + 0.38 * br;
    col[0] = col[1] = col[2] = (float)sw;
  } else if (cls == 2) {
    double cl = 0.22 + 0.78 * br;
    if (c.spinCue) cl *= 0.85 + 0.15 * cos((double)__ldg(P.pPh + p));
    col[0] = (float)(0.76 * cl); col[1] = (float)(0.85 * cl); col[2] = (float)cl;
  } else {
    double t = c.useTemp ? (double)__ldg(P.pT + p) : 0.32;
    if (t < 0) t = 0; else if (t > 1) t = 1;
    double w = t > 0 ? exp(1.4 * log(t)) : 0;       // Math.pow(t, 1.4), t in [0, 1]
    double cr = c.water[0] * (0.9 + 0.1 * w), cg = c.water[1], cb = c.water[2];
    if (f == 1 || f == 4) { cr = cr * 0.45 + 0.55; cg = cg * 0.45 + 0.55; cb = cb * 0.45 + 0.55; }
    double b = (cls == 0 && sunnyBead) ? 1 : br;
    col[0] = (float)(cr * b); col[1] = (float)(cg * b); col[2] = (float)(cb * b);
  }
}

__global__ void __launch_bounds__(kThreads, 3) k_rp_classify(RenderCfg c, PartsDev P, uint8_t* cls, float* d2,
                                                             unsigned* red, int nb) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int n = P.nP;
  unsigned cnt[5] = { 0, 0, 0, 0, 0 };
  unsigned dmin = 0xFFFFFFFFu, dmax = 0, wmin[3] = { ~0u, ~0u, ~0u }, wmax[3] = { 0, 0, 0 };
  constexpr int kHoist = 4;                          // rounds whose inputs are loaded together
  for (int b = blockIdx.x; b < nb; b += gridDim.x) {
    const int base = b * kChunk + w * (kRounds * 32);
    for (int r0 = 0; r0 < kRounds; r0 += kHoist) {
      int fr[kHoist];
      float xr[kHoist], yr[kHoist], zr[kHoist];
#pragma unroll
      for (int i = 0; i < kHoist; i++) {
        int p = base + (r0 + i) * 32 + lane;
        bool v = p < n;
        fr[i] = v ? __ldg(P.pflag + p) : -1;
        xr[i] = v ? __ldg(P.px + p) : 0.f; yr[i] = v ? __ldg(P.py + p) : 0.f; zr[i] = v ? __ldg(P.pz + p) : 0.f;
      }
#pragma unroll
      for (int i = 0; i < kHoist; i++) {
        int p = base + (r0 + i) * 32 + lane;
        if (fr[i] < 0) continue;
        bool sunny;
        int k = rp_class(c, fr[i], xr[i], yr[i], zr[i], P.pDepth + p, &sunny);
        if (k >= 0) {
          float d = dist2(c, xr[i], yr[i], zr[i]);
          d2[p] = d;
          unsigned u = __float_as_uint(d);
          dmin = min(dmin, u); dmax = max(dmax, u);
          for (int j = 0; j < 5; j++) cnt[j] += (k == j);
        }
        cls[p] = k < 0 ? kCulled : (uint8_t)(k | (sunny ? kSunny : 0));
      }
    }
    if (c.spinCol) {
#pragma unroll 4
      for (int r = 0; r < kRounds; r++) {
        int p = base + r * 32 + lane;
        if (p >= n) continue;
        unsigned a = ord_of(__ldg(P.pWx + p)), bb = ord_of(__ldg(P.pWy + p)), e = ord_of(__ldg(P.pWz + p));
        wmin[0] = min(wmin[0], a); wmax[0] = max(wmax[0], a);
        wmin[1] = min(wmin[1], bb); wmax[1] = max(wmax[1], bb);
        wmin[2] = min(wmin[2], e); wmax[2] = max(wmax[2], e);
      }
    }
  }
  const unsigned full = 0xFFFFFFFFu;
  __shared__ unsigned wred[kWarps][R_WORDS];
  for (int j = 0; j < 5; j++) cnt[j] = __reduce_add_sync(full, cnt[j]);
  dmin = __reduce_min_sync(full, dmin); dmax = __reduce_max_sync(full, dmax);
  if (c.spinCol)
    for (int d = 0; d < 3; d++) { wmin[d] = __reduce_min_sync(full, wmin[d]); wmax[d] = __reduce_max_sync(full, wmax[d]); }
  if (lane == 0) {
    for (int j = 0; j < 5; j++) wred[w][R_CNT + j] = cnt[j];
    wred[w][R_DMAX] = dmax; wred[w][R_DMIN] = dmin;
    for (int d = 0; d < 3; d++) { wred[w][R_WMIN + d] = wmin[d]; wred[w][R_WMAX + d] = wmax[d]; }
  }
  __syncthreads();
  // one atomic per word per block
  const int t = threadIdx.x;
  if (t < R_WORDS && (c.spinCol || (t != R_WMAX && t != R_WMAX + 1 && t != R_WMAX + 2 && t < R_WMIN))) {
    unsigned v = wred[0][t];
    for (int j = 1; j < kWarps; j++) {
      unsigned x = wred[j][t];
      if (t < R_WMAX) v += x;
      else if (t == R_DMIN || t >= R_WMIN) v = min(v, x);
      else v = max(v, x);
    }
    if (t < R_WMAX) { if (v) atomicAdd(&red[t], v); }
    else if (t == R_DMIN || t >= R_WMIN) { if (v != 0xFFFFFFFFu) atomicMin(&red[t], v); }
    else if (v) atomicMax(&red[t], v);
  }
}

__global__ void __launch_bounds__(kThreads) k_rp_hist(RenderCfg c, const uint8_t* cls, const float* d2, int n,
                                                      const unsigned* red, int* hist, int nb) {
  __shared__ int sh[kKeys];
  double lo, inv;
  bucket_scale(c, red, &lo, &inv);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int b = blockIdx.x; b < nb; b += gridDim.x) {
    for (int k = threadIdx.x; k < kKeys; k += kThreads) sh[k] = 0;
    __syncthreads();
    const int base = b * kChunk + w * (kRounds * 32);
    int key[kRounds];
#pragma unroll
    for (int r = 0; r < kRounds; r++) {
      int p = base + r * 32 + lane;
      int k = p < n ? __ldg(cls + p) : kCulled;
      float d = p < n ? __ldg(d2 + p) : 0.f;
      key[r] = k != kCulled ? key_of(k & 7, d, lo, inv) : -1;
    }
#pragma unroll
    for (int r = 0; r < kRounds; r++) {
      unsigned peers = __match_any_sync(0xFFFFFFFFu, key[r]);
      if (key[r] >= 0 && (peers & ((1u << lane) - 1)) == 0) atomicAdd(&sh[key[r]], __popc(peers));
    }
    __syncthreads();
    for (int k = threadIdx.x; k < kKeys; k += kThreads) hist[(size_t)k * nb + b] = sh[k];
    __syncthreads();
  }
}

// exclusive scan of one key's row of chunk counts (nb ints, in place) per
// block; the row total goes to totals[key]
__global__ void __launch_bounds__(kThreads) k_rp_scan(int* hist, int nb, int* totals) {
  __shared__ int ws[kWarps];
  int* row = hist + (size_t)blockIdx.x * nb;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  int carry = 0;
  for (int b0 = 0; b0 < nb; b0 += 4 * kThreads) {
    int v[4], s = 0;
    for (int i = 0; i < 4; i++) { int j = b0 + 4 * t + i; v[i] = j < nb ? row[j] : 0; s += v[i]; }
    int x = s;
    for (int o = 1; o < 32; o <<= 1) { int y = __shfl_up_sync(0xFFFFFFFFu, x, o); if (lane >= o) x += y; }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    int before = 0, all = 0;
    for (int j = 0; j < kWarps; j++) { int y = ws[j]; before += j < w ? y : 0; all += y; }
    int run = carry + before + x - s;
    for (int i = 0; i < 4; i++) { int j = b0 + 4 * t + i; if (j < nb) row[j] = run; run += v[i]; }
    carry += all;
    __syncthreads();
  }
  if (t == 0) totals[blockIdx.x] = carry;
}

__global__ void __launch_bounds__(kThreads) k_rp_emit(RenderCfg c, PartsDev P, const uint8_t* cls, const float* d2,
                                                      const unsigned* red, const int* off, const int* totals, int nb,
                                                      RenderOut o) {
  __shared__ int cnt[kWarps][kKeys];
  __shared__ int keyBase[kKeys];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int n = P.nP, base = blockIdx.x * kChunk + w * (kRounds * 32);
  const unsigned full = 0xFFFFFFFFu, lt = (1u << lane) - 1;
  for (int i = threadIdx.x; i < kWarps * kKeys; i += kThreads) (&cnt[0][0])[i] = 0;
  if (w == 0) {                       // exclusive prefix of the 320 key totals, 10 keys a lane
    constexpr int per = kKeys / 32;
    int v[per], s = 0;
    for (int i = 0; i < per; i++) { v[i] = totals[lane * per + i]; s += v[i]; }
    int x = s;
    for (int o = 1; o < 32; o <<= 1) { int y = __shfl_up_sync(full, x, o); if (lane >= o) x += y; }
    int run = x - s;
    for (int i = 0; i < per; i++) { keyBase[lane * per + i] = run; run += v[i]; }
  }
  __syncthreads();
  double lo, inv;
  bucket_scale(c, red, &lo, &inv);
  const Spin sp = c.spinCol ? spin_scale(red) : Spin{};
  for (int b = blockIdx.x; b < nb; b += gridDim.x) {
    const int base = b * kChunk + w * (kRounds * 32);
    // the keys of the warp's 256 particles, loaded once and kept in registers
    int key[kRounds];
    unsigned sunnyBits = 0;
#pragma unroll
    for (int r = 0; r < kRounds; r++) {
      int p = base + r * 32 + lane;
      int k = p < n ? __ldg(cls + p) : kCulled;
      float d = p < n ? __ldg(d2 + p) : 0.f;        // stale for a culled particle, unused
      key[r] = k != kCulled ? key_of(k & 7, d, lo, inv) : -1;
      sunnyBits |= (k != kCulled && (k & kSunny)) ? 1u << r : 0u;
    }
    // per-warp key counts in particle order
#pragma unroll
    for (int r = 0; r < kRounds; r++) {
      unsigned peers = __match_any_sync(full, key[r]);
      if (key[r] >= 0 && (peers & lt) == 0) cnt[w][key[r]] += __popc(peers);
      __syncwarp();
    }
    __syncthreads();
    // chunk offset of every key, then the warps' shares in particle order
    for (int k = threadIdx.x; k < kKeys; k += kThreads) {
      int run = keyBase[k] + off[(size_t)k * nb + b];
      for (int j = 0; j < kWarps; j++) { int t = cnt[j][k]; cnt[j][k] = run; run += t; }
    }
    __syncthreads();
    // draw-list slots of all rounds first, so that the loads below are not
    // held behind warp synchronisation
    int slot[kRounds];
#pragma unroll
    for (int r = 0; r < kRounds; r++) {
      unsigned peers = __match_any_sync(full, key[r]);
      slot[r] = key[r] >= 0 ? cnt[w][key[r]] + __popc(peers & lt) : 0;
      __syncwarp();
      if (key[r] >= 0 && (peers & lt) == 0) cnt[w][key[r]] += __popc(peers);
      __syncwarp();
    }
#pragma unroll
    for (int r = 0; r < kRounds; r++) {
      if (key[r] < 0) continue;
      const int p = base + r * 32 + lane, k = slot[r];
      const int cl = key[r] % 5, f = __ldg(P.pflag + p);
      const float x = __ldg(P.px + p), y = __ldg(P.py + p), z = __ldg(P.pz + p);
      const bool sunny = (sunnyBits >> r) & 1;
      float col[3];
      rp_color(c, P, p, cl, f, sunny, x, y, z, sp, col);
      const size_t k3 = 3 * (size_t)k;
      o.pos[k3] = x; o.pos[k3 + 1] = y; o.pos[k3 + 2] = z;
      o.col[k3] = col[0]; o.col[k3 + 1] = col[1]; o.col[k3 + 2] = col[2];
      o.alpha[k] = c.alpha[cl]; o.size[k] = c.size[cl]; o.sprite[k] = c.sprite[cl];
    }
    __syncthreads();                                 // the counters are reset for the next chunk
    for (int i = threadIdx.x; i < kWarps * kKeys; i += kThreads) (&cnt[0][0])[i] = 0;
    __syncthreads();
  }
}

}  // namespace

size_t render_scratch_bytes(long long capacity) {
  size_t nb = (size_t)((capacity + kChunk - 1) / kChunk);
  return sizeof(unsigned) * 16 + sizeof(int) * kKeys * ((nb ? nb : 1) + 1) + sizeof(float) * capacity + capacity;
}

// the counts come back through red[0..4]; the caller reads them after the
// stream drains
void launch_render_particles(const RenderCfg& c, const PartsDev& P, void* scratch, RenderOut o, cudaStream_t s) {
  const int n = P.nP, nb = (n + kChunk - 1) / kChunk;
  unsigned* red = (unsigned*)scratch;
  int* totals = (int*)(red + 16);
  int* hist = totals + kKeys;
  float* d2 = (float*)(hist + (size_t)kKeys * (nb ? nb : 1));
  uint8_t* cls = (uint8_t*)(d2 + n);
  cudaMemsetAsync(red, 0, sizeof(unsigned) * R_DMIN, s);
  cudaMemsetAsync(red + R_DMIN, 0xFF, sizeof(unsigned) * (R_WORDS - R_DMIN), s);
  if (!n) return;
  static int occ[3] = { 0, 0, 0 }, sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[0], k_rp_classify, kThreads, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[1], k_rp_hist, kThreads, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[2], k_rp_emit, kThreads, 0);
  }
  auto grid = [&](int i) { return std::max(1, std::min(nb, sms * std::max(occ[i], 1))); };
  k_rp_classify<<<grid(0), kThreads, 0, s>>>(c, P, cls, d2, red, nb);
  k_rp_hist<<<grid(1), kThreads, 0, s>>>(c, cls, d2, n, red, hist, nb);
  k_rp_scan<<<kKeys, kThreads, 0, s>>>(hist, nb, totals);
  k_rp_emit<<<grid(2), kThreads, 0, s>>>(c, P, cls, d2, red, hist, totals, nb, o);
}
