// ws_sor_tb.cu — the pressure solve of _pressureSolve (js/solver.js:1368-1404)
// on every SM at once: red-black SOR with temporal blocking.
//
// Partition. The grid is cut into 4x4x4-cell bricks. Bricks holding a fluid
// cell are taken in Morton order and split into one contiguous chunk per CTA
// with equal shares of weight (interior fluid cells plus kBrickWeight per
// brick), so each CTA owns a compact patch of the ocean shell (about 700
// cells at 128^3).
//
// Region. A CTA keeps in shared memory its owned bricks plus every active
// brick among their 26 neighbours, densely (64 q values per brick). The
// interior fluid cells of the region are labelled with d, their L1 distance
// in cells to the boxes of the owned bricks (d = 0 owned). d changes by at
// most one between neighbouring cells, and a red-black half-sweep only
// propagates information one cell, so after loading exact values for d <= 4,
// the CTA can run four half-sweeps (two iterations) on its own: half-sweep t
// updates the cells with d <= 4 - t, and after the fourth the owned cells
// hold exactly the values of the global sweep. Each cell's update reads the same six neighbours in
// the same order with the same arithmetic as the reference's sweep, so the
// iterates are bitwise those of the plain red-black solve.
//
// Exchange. After each such epoch e a CTA writes its owned cells into one of
// two global exchange buffers (e & 1) as 64-bit words (q's bits | e << 32),
// one single-copy-atomic relaxed store per cell and no fence or flag; before
// the next epoch every thread loads its halo cells from that buffer and
// polls a word again until its tag reads e. The tag travels in the same word
// as the value, so a matching tag proves the value, and a CTA waits only for
// the values it needs. Double buffering makes the write of epoch e + 2 safe
// against neighbours still reading epoch e: a CTA computes epoch e + 2 only
// after reading its neighbours' epoch e + 1 values, which each neighbour
// wrote after it had read this CTA's epoch e values (halo adjacency is
// symmetric). The plan phase clears the tags of every owned cell in both
// buffers before the first epoch, so stale words of an earlier solve never
// match.
//
// Residual check. Every sorCheckEvery iterations (epochs end on check
// iterations) the FP64 partial ||b - A q||^2 and ||b||^2 of the owned cells
// is published, all CTAs wait for all partials (a counter) and sum them in
// CTA order, so every CTA takes the same stop decision. Partials alternate
// between two buffers so a CTA running ahead cannot overwrite one that a
// slower CTA still sums.
//
// The plan (brick counts, Morton scan, chunks, regions) is built inside the
// same cooperative launch, separated by three grid barriers. When a region
// does not fit in shared memory, every CTA takes the same fallback: the
// red-black sweep over its owned bricks in global memory with a grid barrier
// per half-sweep (same arithmetic, same iterates).
//
// Every wait is bounded: after kTbSpinLimit polls the CTA latches
// WS_DERR_TIMEOUT, stops, and the waits of the others run out in turn. The
// cooperative launch guarantees that all CTAs are resident, so a healthy
// run never reaches the limit.
#include "ws_kernels.cuh"
#include <algorithm>

namespace {

constexpr int kTbThreads = 1024;
constexpr int kRbMax = 256;                 // region bricks per CTA
constexpr int kEMax = 4096;                 // update entries (d <= 3) per CTA
constexpr int kLMax = 4096;                 // halo reload cells (1 <= d <= 4) per CTA
constexpr int kOMax = 2048;                 // owned interior fluid cells per CTA
constexpr int kHashSlots = 1024;            // open-addressing table of region bricks
constexpr int kZero = kRbMax * 64;          // dense index of the always-zero cell
constexpr long long kTbSpinLimit = 4000000LL;
constexpr int kMaxCtas = 1024;
// Chunk weight of an active brick: its interior fluid cells plus this much.
// Equal shares of fluid alone gave CTAs 13-55 owned bricks at 128^3 (bricks
// at the shell's edges hold few fluid cells), and the CTA with the most
// bricks has the largest region, which every other CTA waits for at the end
// of the plan; the per-brick term evens out the brick counts too.
constexpr int kBrickWeight = 16;

// device control block, zeroed before every solve
struct TbCtl {
  unsigned barCount, barGen;     // grid barrier
  unsigned resCount;             // residual partials published so far (all checks)
  int overflow;                  // some region did not fit: every CTA takes the fallback
  int pad[12];
};

struct TbArgs {
  Dims d;
  float* q;                      // the solve's q (epochs 0, 2, 4, ... end here)
  unsigned long long* xq;        // exchange: two buffers of nCells words (q bits | epoch << 32)
  const float* rhs;
  const float* pw;               // omega/diag, negative off the fluid
  const uint8_t* diag8;
  int nbx, nby, nbz, mbits;      // bricks per axis; Morton cube side 2^mbits
  int* brickW;                   // per Morton code: chunk weight (interior fluid + kBrickWeight) | any-fluid << 8
  int2* cntPart;                 // per CTA: (active bricks, interior fluid cells) of its Morton chunk
  int* actLin;                   // active brick t -> linear brick index
  int* actWPre;                  // active brick t -> chunk weight before it
  int* brickOrd;                 // linear brick -> active ordinal, -1 inactive
  int* chunkStart;               // CTA -> first owned active brick ([P] = number of active bricks)
  double2* resPart;              // 2 x P residual partials
  TbCtl* ctl;
  double om1;
  int iters, check;
  double tol;
  int* err;
  int* outIters;
  double* outRel;
  int* outPath;
};

// shared-memory layout (dynamic)
struct TbSmem {
  float q[kRbMax * 64 + 4];               // dense region q; [kZero] = 0
  uint8_t dist[kRbMax * 64];              // 0..4 distance d, 5 farther, 254 constant
  int hkey[kHashSlots];
  short hval[kHashSlots];
  int rbLin[kRbMax];
  short rbX[kRbMax], rbY[kRbMax], rbZ[kRbMax];   // brick coordinates of each slot
  short rbOwn[kRbMax];
  short rbNb[kRbMax][6];
  unsigned rbOwnMask[kRbMax];             // which of the 27 bricks around a slot (itself included) this CTA owns
  unsigned short eSelf[kEMax];
  unsigned eNb[kEMax][3];                 // six neighbour dense indices, two per word
  float eRhs[kEMax], ePw[kEMax];
  unsigned short lDense[kLMax];
  unsigned lGlob[kLMax];
  unsigned oGlob[kOMax];                  // global index of each owned entry (buckets 0 and 4, in order)
};

__device__ __forceinline__ unsigned compact1by2(unsigned x) {
  x &= 0x09249249u;
  x = (x ^ (x >> 2)) & 0x030c30c3u;
  x = (x ^ (x >> 4)) & 0x0300f00fu;
  x = (x ^ (x >> 8)) & 0xff0000ffu;
  x = (x ^ (x >> 16)) & 0x000003ffu;
  return x;
}
__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" :: "l"(p), "l"(v) : "memory");
}

// bounded grid barrier on ctl->barCount/barGen; false when a wait timed out
__device__ bool tb_grid_barrier(TbCtl* ctl, int* err, int* sAbort) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* vgen = &ctl->barGen;
    unsigned g = *vgen;
    __threadfence();
    if (atomicAdd(&ctl->barCount, 1u) == gridDim.x - 1) {
      atomicExch(&ctl->barCount, 0u);
      __threadfence();
      atomicAdd(&ctl->barGen, 1u);
    } else {
      long long n = 0;
      while (*vgen == g) {
        if (++n > kTbSpinLimit) { atomicOr(err, WS_DERR_TIMEOUT); *sAbort = 1; break; }
      }
    }
    __threadfence();
    if (*(volatile int*)err & WS_DERR_TIMEOUT) *sAbort = 1;
  }
  __syncthreads();
  return *(volatile int*)sAbort == 0;
}

// the CTA that owns an active brick with chunk weight `wpre` before
// it in Morton order (NF: the total weight)
__device__ __forceinline__ int owner_of(long long wpre, int P, long long NF) {
  if (NF <= 0) return 0;
  long long o = wpre * P / NF;
  return (int)(o < P - 1 ? o : P - 1);
}
__device__ __forceinline__ bool interior(const Dims& d, int i, int j, int k) {
  return i >= 1 && j >= 1 && k >= 1 && i + 2 <= d.nx && j + 2 <= d.ny && k + 2 <= d.nz;
}

// dense neighbour (direction 0..5 = -x, +x, -y, +y, -z, +z) of dense cell x
__device__ __forceinline__ int dense_nb(const TbSmem& S, int x, int dir) {
  const int s = x >> 6, c = x & 63, cx = c & 3, cy = (c >> 2) & 3, cz = c >> 4;
  int nbS;
  switch (dir) {
    case 0: if (cx > 0) return x - 1; nbS = S.rbNb[s][0]; return nbS < 0 ? kZero : (nbS << 6) | (c + 3);
    case 1: if (cx < 3) return x + 1; nbS = S.rbNb[s][1]; return nbS < 0 ? kZero : (nbS << 6) | (c - 3);
    case 2: if (cy > 0) return x - 4; nbS = S.rbNb[s][2]; return nbS < 0 ? kZero : (nbS << 6) | (c + 12);
    case 3: if (cy < 3) return x + 4; nbS = S.rbNb[s][3]; return nbS < 0 ? kZero : (nbS << 6) | (c - 12);
    case 4: if (cz > 0) return x - 16; nbS = S.rbNb[s][4]; return nbS < 0 ? kZero : (nbS << 6) | (c + 48);
    default: if (cz < 3) return x + 16; nbS = S.rbNb[s][5]; return nbS < 0 ? kZero : (nbS << 6) | (c - 48);
  }
}
// global cell index of dense cell x (region brick s holds linear brick rbLin[s]);
// false outside the domain
__device__ __forceinline__ bool dense_global(const TbArgs& a, const TbSmem& S, int x, unsigned& g, int& i, int& j,
                                             int& k) {
  const int s = x >> 6, c = x & 63;
  i = S.rbX[s] * 4 + (c & 3); j = S.rbY[s] * 4 + ((c >> 2) & 3); k = S.rbZ[s] * 4 + (c >> 4);
  if (i >= a.d.nx || j >= a.d.ny || k >= a.d.nz) return false;
  g = ((unsigned)k * (unsigned)a.d.ny + (unsigned)j) * (unsigned)a.d.nx + (unsigned)i;
  return true;
}

__device__ __forceinline__ bool hash_insert(TbSmem& S, int key, int* nRegion, int* sOverflow, int fixedSlot,
                                            short owner, int nbx, int nby) {
  unsigned h = ((unsigned)key * 2654435761u) >> 22;          // 10 bits
  for (int probe = 0; probe < kHashSlots; probe++, h = (h + 1) & (kHashSlots - 1)) {
    int prev = atomicCAS(&S.hkey[h], -1, key);
    if (prev == -1) {
      int slot = fixedSlot >= 0 ? fixedSlot : atomicAdd(nRegion, 1);
      S.hval[h] = (short)(slot < kRbMax ? slot : -1);
      if (slot < kRbMax) {
        S.rbLin[slot] = key; S.rbOwn[slot] = owner;
        const int t = key / nbx;
        S.rbX[slot] = (short)(key - t * nbx); S.rbY[slot] = (short)(t % nby); S.rbZ[slot] = (short)(t / nby);
      }
      else *sOverflow = 1;
      return true;
    }
    if (prev == key) return false;
  }
  *sOverflow = 1;
  return false;
}
__device__ __forceinline__ int hash_find(const TbSmem& S, int key) {
  unsigned h = ((unsigned)key * 2654435761u) >> 22;
  for (int probe = 0; probe < kHashSlots; probe++, h = (h + 1) & (kHashSlots - 1)) {
    int k = S.hkey[h];
    if (k == key) return S.hval[h];
    if (k == -1) return -1;
  }
  return -1;
}

// block-wide exclusive scan of two ints (1024 threads); totals returned
__device__ __forceinline__ int2 block_scan2(int a, int b, int2& total, int2* sw) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int xa = a, xb = b;
  for (int o = 1; o < 32; o <<= 1) {
    int ya = __shfl_up_sync(0xffffffffu, xa, o), yb = __shfl_up_sync(0xffffffffu, xb, o);
    if (lane >= o) { xa += ya; xb += yb; }
  }
  if (lane == 31) sw[wid] = make_int2(xa, xb);
  __syncthreads();
  if (wid == 0) {
    int2 v = lane < (int)(blockDim.x >> 5) ? sw[lane] : make_int2(0, 0);
    int ca = v.x, cb = v.y;
    for (int o = 1; o < 32; o <<= 1) {
      int ya = __shfl_up_sync(0xffffffffu, ca, o), yb = __shfl_up_sync(0xffffffffu, cb, o);
      if (lane >= o) { ca += ya; cb += yb; }
    }
    sw[lane] = make_int2(ca - v.x, cb - v.y);            // exclusive warp offsets
    if (lane == 31) sw[32] = make_int2(ca, cb);
  }
  __syncthreads();
  int2 base = sw[wid];
  total = sw[32];
  int2 r = make_int2(base.x + xa - a, base.y + xb - b);
  __syncthreads();                                         // sw reusable
  return r;
}

// one cell update of the reference's sweep (js/solver.js:1397-1404; sor_update)
__device__ __forceinline__ float relax(float qc, float pw, float rhs, const float* v, double om1) {
  return sor_update(qc, pw, rhs, v[0], v[1], v[2], v[3], v[4], v[5], om1);
}

// residual partial of the owned cells (dense order, deterministic) of the
// state in S.q; block total returned on thread 0
__device__ double2 owned_residual(const TbArgs& a, const TbSmem& S, int O, double2* sred) {
  double rr = 0, bb = 0;
  for (int x = threadIdx.x; x < O * 64; x += blockDim.x) {
    if (S.dist[x] != 0) continue;
    unsigned g; int i, j, k;
    dense_global(a, S, x, g, i, j, k);
    float v[6];
#pragma unroll
    for (int dir = 0; dir < 6; dir++) v[dir] = S.q[dense_nb(S, x, dir)];
    double sum = (double)v[0];
    sum += (double)v[1]; sum += (double)v[2]; sum += (double)v[3]; sum += (double)v[4]; sum += (double)v[5];
    double b = a.rhs[g];
    double r = b + sum - (double)a.diag8[g] * (double)S.q[x];
    rr += r * r; bb += b * b;
  }
  rr = warp_sum(rr); bb = warp_sum(bb);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sred[wid] = make_double2(rr, bb);
  __syncthreads();
  double2 out = make_double2(0, 0);
  if (wid == 0) {
    double2 v = lane < (int)(blockDim.x >> 5) ? sred[lane] : make_double2(0, 0);
    rr = warp_sum(v.x); bb = warp_sum(v.y);
    out = make_double2(rr, bb);
  }
  __syncthreads();
  return out;
}

// publish this CTA's partial for check number k, wait for all, sum in a
// fixed order (lane l adds partials l, l + 32, ..., then a fixed butterfly);
// every CTA gets the same value. false when the wait timed out.
__device__ bool global_residual(const TbArgs& a, double2 part, int k, double* sRel, int* sAbort) {
  const int P = gridDim.x;
  double2* buf = a.resPart + (size_t)(k & 1) * P;
  if (threadIdx.x == 0) {
    __stcg(&buf[blockIdx.x], part);
    fence_acq_rel_gpu();
    atomicAdd(&a.ctl->resCount, 1u);
    if (!bounded_wait_geq(&a.ctl->resCount, (unsigned)P * (unsigned)(k + 1), kTbSpinLimit, a.err)) *sAbort = 1;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    double rr = 0, bb = 0;
    if (!*(volatile int*)sAbort)
      for (int b = threadIdx.x; b < P; b += 32) { const double2 v = __ldcg(&buf[b]); rr += v.x; bb += v.y; }
    for (int o = 16; o > 0; o >>= 1) {
      rr += __shfl_xor_sync(0xffffffffu, rr, o);
      bb += __shfl_xor_sync(0xffffffffu, bb, o);
    }
    if (threadIdx.x == 0) *sRel = bb > 0 ? sqrt(rr) / sqrt(bb) : sqrt(rr);
  }
  __syncthreads();
  return *(volatile int*)sAbort == 0;
}

}  // namespace


extern __shared__ __align__(16) unsigned char tb_smem_raw[];

// The whole solve in one cooperative launch of one 1024-thread CTA per SM.
__global__ void __launch_bounds__(kTbThreads, 1) k_sor_tb(TbArgs a) {
  TbSmem& S = *reinterpret_cast<TbSmem*>(tb_smem_raw);
  __shared__ int sAbort, sOverflow, nRegion, nReload, sT0, sT1, sA;
  __shared__ int bucket[8], bstart[8], bcur[8];
  __shared__ int2 sScan[33];
  __shared__ double2 sRed[32];
  __shared__ double sRel;
  __shared__ long long sNF;
  const int P = gridDim.x, p = blockIdx.x, tid = threadIdx.x, T = blockDim.x;
  const int lane = tid & 31;
  const Dims& d = a.d;
  int it = 0, O = 0, R = 0, path = 3;
  double rel = -1;
  if (tid == 0) { sAbort = 0; sOverflow = 0; nRegion = 0; nReload = 0; }
  if (tid < 8) bucket[tid] = 0;
  __syncthreads();

  // ---- phase 0: interior fluid cells per brick, Morton order, one chunk of codes per CTA
  const long long MC = 1LL << (3 * a.mbits);
  const long long per = (MC + P - 1) / P;
  const long long c0 = std::min(MC, (long long)p * per), c1 = std::min(MC, c0 + per);
  if (p == 0) {
    for (int q = tid; q <= P; q += T) a.chunkStart[q] = q == 0 ? 0 : 0x7fffffff;
  }
  {
    int actSum = 0, wSum = 0;
    const bool vec = (d.nx & 3) == 0;
    for (long long base = c0 * 16; base < c1 * 16; base += T) {
      // 16 consecutive threads share one brick: one row of 4 cells each
      const long long item = base + tid, m = item >> 4;
      int w = 0, act = 0;
      if (m < c1) {
        const int row = (int)(item & 15);
        const unsigned bx = compact1by2((unsigned)m), by = compact1by2((unsigned)(m >> 1)),
                       bz = compact1by2((unsigned)(m >> 2));
        const int j = (int)by * 4 + (row & 3), k = (int)bz * 4 + (row >> 2), i0 = (int)bx * 4;
        if ((int)bx < a.nbx && (int)by < a.nby && (int)bz < a.nbz && j < d.ny && k < d.nz) {
          const long long g = ((long long)k * d.ny + j) * d.nx + i0;
          float v[4];
          if (vec) {
            const float4 f = __ldcg(reinterpret_cast<const float4*>(a.pw + g));
            v[0] = f.x; v[1] = f.y; v[2] = f.z; v[3] = f.w;
          } else {
#pragma unroll
            for (int c = 0; c < 4; c++) v[c] = i0 + c < d.nx ? __ldcg(a.pw + g + c) : -1.f;
          }
#pragma unroll
          for (int c = 0; c < 4; c++)
            if (v[c] >= 0.f) { act = 1; if (interior(d, i0 + c, j, k)) w++; }
        }
      }
      // the 16 rows of a brick sit in one half-warp
      for (int o = 8; o > 0; o >>= 1) {
        w += __shfl_down_sync(0xffffffffu, w, o, 16);
        act |= __shfl_down_sync(0xffffffffu, act, o, 16);
      }
      if ((tid & 15) == 0 && m < c1) {
        w += act * kBrickWeight;
        a.brickW[m] = w | (act << 8);
        actSum += act; wSum += w;
      }
    }
    actSum = warp_sum(actSum); wSum = warp_sum(wSum);
    if (lane == 0) sScan[tid >> 5] = make_int2(actSum, wSum);
    __syncthreads();
    if (tid < 32) {
      int2 v = tid < (T >> 5) ? sScan[tid] : make_int2(0, 0);
      v.x = warp_sum(v.x); v.y = warp_sum(v.y);
      if (tid == 0) __stcg(&a.cntPart[p], v);
    }
  }
  if (!tb_grid_barrier(a.ctl, a.err, &sAbort)) goto done;

  // ---- phase 1: ordinals and fluid prefixes of this chunk's active bricks,
  // the dense brick -> ordinal map, and the CTA chunk starts
  {
    if (tid < 32) {
      long long bA = 0, bW = 0, tA = 0, tW = 0;
      for (int b = tid; b < P; b += 32) {
        const int2 v = __ldcg(&a.cntPart[b]);
        if (b < p) { bA += v.x; bW += v.y; }
        tA += v.x; tW += v.y;
      }
      bA = warp_sum(bA); bW = warp_sum(bW); tA = warp_sum(tA); tW = warp_sum(tW);
      if (tid == 0) { sT0 = (int)bA; sT1 = (int)bW; sA = (int)tA; sNF = tW; }
    }
    __syncthreads();
    int baseA = sT0, baseW = sT1;
    const int A = sA;
    const long long NF = sNF;
    for (long long m0 = c0; m0 < c1; m0 += T) {
      const long long m = m0 + tid;
      const int v = m < c1 ? __ldcg(&a.brickW[m]) : 0;
      const int act = (v >> 8) & 1, w = v & 255;
      int2 tot;
      const int2 ex = block_scan2(act, w, tot, sScan);
      if (m < c1) {
        const unsigned bx = compact1by2((unsigned)m), by = compact1by2((unsigned)(m >> 1)),
                       bz = compact1by2((unsigned)(m >> 2));
        if ((int)bx < a.nbx && (int)by < a.nby && (int)bz < a.nbz) {
          const int lin = ((int)bz * a.nby + (int)by) * a.nbx + (int)bx;
          if (act) {
            const int t = baseA + ex.x;
            const long long wpre = baseW + ex.y;
            a.actLin[t] = lin; a.actWPre[t] = (int)wpre; a.brickOrd[lin] = t;
            // the next active brick starts every CTA q whose first fluid cell
            // (prefix ceil(q NF / P)) lies in (wpre, wpre + w]
            if (w > 0) {
              const long long qlo = wpre * P / NF + 1, qhi = std::min((long long)P - 1, (wpre + w) * P / NF);
              for (long long q = qlo; q <= qhi; q++) a.chunkStart[q] = t + 1;
            }
            if (t == A - 1) a.chunkStart[P] = A;
          } else {
            a.brickOrd[lin] = -1;
          }
        }
      }
      baseA += tot.x; baseW += tot.y;
    }
  }
  if (!tb_grid_barrier(a.ctl, a.err, &sAbort)) goto done;
  // no fluid cell: the reference returns before its first sweep
  // (js/solver.js:1330); every CTA read the same total, so all leave here
  if (sA == 0) { rel = 0; goto done; }

  // ---- phase 2: this CTA's region
  {
    const int A = sA;
    const long long NF = sNF;
    if (tid == 0) {
      int s0 = __ldcg(&a.chunkStart[p]), s1 = __ldcg(&a.chunkStart[p + 1]);
      if (s0 > A) s0 = A;
      if (s1 > A) s1 = A;
      sT0 = s0; sT1 = s1 > s0 ? s1 : s0;
      nRegion = sT1 - sT0;
      if (nRegion > kRbMax) sOverflow = 1;
    }
    for (int h = tid; h < kHashSlots; h += T) S.hkey[h] = -1;
    __syncthreads();
    const int t0 = sT0;
    O = sT1 - sT0;
    if (!sOverflow) {
      for (int s = tid; s < O; s += T)
        hash_insert(S, __ldcg(&a.actLin[t0 + s]), &nRegion, &sOverflow, s, (short)p, a.nbx, a.nby);
      __syncthreads();
      // the active bricks among the owned bricks' 26 neighbours that other CTAs own
      for (int item = tid; item < O * 26; item += T) {
        const int s = item / 26, n27 = item % 26 < 13 ? item % 26 : item % 26 + 1;
        const int bx = S.rbX[s], by = S.rbY[s], bz = S.rbZ[s];
        const int nx_ = bx + n27 % 3 - 1, ny_ = by + (n27 / 3) % 3 - 1, nz_ = bz + n27 / 9 - 1;
        if (nx_ < 0 || ny_ < 0 || nz_ < 0 || nx_ >= a.nbx || ny_ >= a.nby || nz_ >= a.nbz) continue;
        const int lin2 = (nz_ * a.nby + ny_) * a.nbx + nx_;
        const int ord = __ldcg(&a.brickOrd[lin2]);
        if (ord < 0) continue;
        const int ow = owner_of(__ldcg(&a.actWPre[ord]), P, NF);
        if (ow != p) hash_insert(S, lin2, &nRegion, &sOverflow, -1, (short)ow, a.nbx, a.nby);
      }
      __syncthreads();
      if (tid == 0 && nRegion > kRbMax) sOverflow = 1;
      __syncthreads();
    }
    R = sOverflow ? 0 : nRegion;
    // face neighbours of each region brick (slot, or -1: outside the region),
    // and which of its 27 surrounding bricks this CTA owns
    for (int item = tid; item < R * 6; item += T) {
      const int s = item / 6, dir = item % 6;
      int bx = S.rbX[s], by = S.rbY[s], bz = S.rbZ[s];
      if (dir == 0) bx--; else if (dir == 1) bx++; else if (dir == 2) by--; else if (dir == 3) by++;
      else if (dir == 4) bz--; else bz++;
      int slot = -1;
      if (bx >= 0 && by >= 0 && bz >= 0 && bx < a.nbx && by < a.nby && bz < a.nbz)
        slot = hash_find(S, (bz * a.nby + by) * a.nbx + bx);
      S.rbNb[s][dir] = (short)slot;
    }
    for (int s = tid; s < R; s += T) S.rbOwnMask[s] = 0;
    __syncthreads();
    for (int item = tid; item < (R - O) * 27; item += T) {
      const int s = O + item / 27, n27 = item % 27;
      const int bx = S.rbX[s] + n27 % 3 - 1, by = S.rbY[s] + (n27 / 3) % 3 - 1, bz = S.rbZ[s] + n27 / 9 - 1;
      if (bx < 0 || by < 0 || bz < 0 || bx >= a.nbx || by >= a.nby || bz >= a.nbz) continue;
      const int slot = hash_find(S, (bz * a.nby + by) * a.nbx + bx);
      if (slot >= 0 && slot < O) atomicOr(&S.rbOwnMask[s], 1u << n27);
    }
    __syncthreads();
    // dense q of the region and the cell states: 0..4 the distance d of an
    // interior fluid cell (5: farther), 254 constant (no interior fluid:
    // never updated). One thread per 4-cell brick row (float4 loads when rows
    // are 16-byte aligned), four rows in flight per thread.
    // Update entries are counted per bucket (colour, d <= 3) here, two
    // 8-bit counters per byte lane of two words per thread (at most 16 cells
    // per bucket and pass, since R * 16 rows <= 4 T), so the bucketing below
    // needs a single pass.
    {
      const bool vec = (d.nx & 3) == 0;
      const int nRows = R * 16;
      unsigned cnt0 = 0u, cnt1 = 0u;         // buckets 0-3 and 4-7, one byte each
      for (int r0 = 0; r0 < nRows; r0 += 4 * T) {
        float qv[4][4], pv[4][4];
        int rowOk[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int row = r0 + u * T + tid;
          rowOk[u] = 0;
#pragma unroll
          for (int c = 0; c < 4; c++) { qv[u][c] = 0.f; pv[u][c] = -1.f; }
          if (row >= nRows) continue;
          const int sl = row >> 4, rr = row & 15;
          const int j = S.rbY[sl] * 4 + (rr & 3), k = S.rbZ[sl] * 4 + (rr >> 2), i0 = S.rbX[sl] * 4;
          if (j >= d.ny || k >= d.nz) continue;
          rowOk[u] = 1;
          const long long g0 = ((long long)k * d.ny + j) * d.nx + i0;
          if (vec) {
            const float4 q4 = __ldcg(reinterpret_cast<const float4*>(a.q + g0));
            const float4 p4 = __ldcg(reinterpret_cast<const float4*>(a.pw + g0));
            qv[u][0] = q4.x; qv[u][1] = q4.y; qv[u][2] = q4.z; qv[u][3] = q4.w;
            pv[u][0] = p4.x; pv[u][1] = p4.y; pv[u][2] = p4.z; pv[u][3] = p4.w;
          } else {
#pragma unroll
            for (int c = 0; c < 4; c++)
              if (i0 + c < d.nx) { qv[u][c] = __ldcg(a.q + g0 + c); pv[u][c] = __ldcg(a.pw + g0 + c); }
          }
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int row = r0 + u * T + tid;
          if (row >= nRows) continue;
          const int sl = row >> 4, rr = row & 15, cy = rr & 3, cz = rr >> 2;
          const unsigned mask = sl < O ? 0u : S.rbOwnMask[sl];
#pragma unroll
          for (int c = 0; c < 4; c++) {
            const int x = row * 4 + c;
            const int i = S.rbX[sl] * 4 + c, j = S.rbY[sl] * 4 + cy, k = S.rbZ[sl] * 4 + cz;
            uint8_t st = 254;
            if (rowOk[u] && i < d.nx && pv[u][c] >= 0.f && interior(d, i, j, k)) {
              if (sl < O) st = 0;
              else {
                // L1 distance to the nearest owned brick box among the 26 around this one
                int best = 5;
                for (unsigned m = mask; m; m &= m - 1) {
                  const int n27 = __ffs(m) - 1, ox = n27 % 3 - 1, oy = (n27 / 3) % 3 - 1, oz = n27 / 9 - 1;
                  const int dd = (ox < 0 ? c + 1 : ox > 0 ? 4 - c : 0) + (oy < 0 ? cy + 1 : oy > 0 ? 4 - cy : 0) +
                                 (oz < 0 ? cz + 1 : oz > 0 ? 4 - cz : 0);
                  best = dd < best ? dd : best;
                }
                st = (uint8_t)best;
              }
              if (st <= 3) {
                const unsigned inc = 1u << (8 * st);
                if ((i + j + k) & 1) cnt1 += inc; else cnt0 += inc;
              }
            }
            S.q[x] = rowOk[u] && i < d.nx ? qv[u][c] : 0.f;
            S.dist[x] = st;
          }
        }
      }
#pragma unroll
      for (int b = 0; b < 8; b++) {
        const int v = warp_sum((int)(((b < 4 ? cnt0 : cnt1) >> (8 * (b & 3))) & 0xffu));
        if (lane == 0 && v) atomicAdd(&bucket[b], v);
      }
    }
    if (tid == 0) S.q[kZero] = 0.f;
    __syncthreads();
    if (tid == 0) {
      int acc = 0;
      for (int b = 0; b < 8; b++) { bstart[b] = acc; bcur[b] = acc; acc += bucket[b]; }
      if (acc > kEMax || bucket[0] + bucket[4] > kOMax) sOverflow = 1;
    }
    __syncthreads();
    // update entries: cells with d <= 3, bucketed by (colour, d), and the
    // halo cells reloaded after every epoch (1 <= d <= 4)
    {
      for (int x0 = 0; x0 < R * 64; x0 += T) {
        const int x = x0 + tid;
        int b = -1;
        bool rl = false;
        unsigned g = 0; int i = 0, j = 0, k = 0;
        if (x < R * 64 && S.dist[x] <= 4) {
          dense_global(a, S, x, g, i, j, k);
          if (S.dist[x] <= 3) b = ((i + j + k) & 1) * 4 + S.dist[x];
          rl = S.dist[x] >= 1;
        }
        const unsigned grp = __match_any_sync(0xffffffffu, b);
        const int leader = __ffs(grp) - 1;
        {
          int base = 0;
          if (b >= 0 && lane == leader) base = atomicAdd(&bcur[b], __popc(grp));
          base = __shfl_sync(0xffffffffu, base, leader);
          if (b >= 0) {
            const int pos = base + __popc(grp & ((1u << lane) - 1u));
            if (pos < kEMax) {
              int nb[6];
#pragma unroll
              for (int dir = 0; dir < 6; dir++) nb[dir] = dense_nb(S, x, dir);
              S.eSelf[pos] = (unsigned short)x;
              S.eNb[pos][0] = (unsigned)nb[0] | ((unsigned)nb[1] << 16);
              S.eNb[pos][1] = (unsigned)nb[2] | ((unsigned)nb[3] << 16);
              S.eNb[pos][2] = (unsigned)nb[4] | ((unsigned)nb[5] << 16);
              if (b == 0 || b == 4) {
                const int o = b == 0 ? pos - bstart[0] : bucket[0] + pos - bstart[4];
                if (o < kOMax) S.oGlob[o] = g;
              }
            }
          }
          const unsigned m = __ballot_sync(0xffffffffu, rl);
          int rbase = 0;
          if (lane == 0 && m) rbase = atomicAdd(&nReload, __popc(m));
          rbase = __shfl_sync(0xffffffffu, rbase, 0);
          if (rl) {
            const int rpos = rbase + __popc(m & ((1u << lane) - 1u));
            if (rpos < kLMax) { S.lDense[rpos] = (unsigned short)x; S.lGlob[rpos] = g; }
          }
        }
      }
      __syncthreads();
    }
    // right-hand side and relaxation weight of every entry, gathered after
    // the bucketing (whose loop carries shuffles and shared atomics) with
    // four loads in flight per thread
    if (!sOverflow) {
      const int nE = bstart[7] + bucket[7];
      for (int e0 = tid; e0 < nE; e0 += 4 * T) {
        float r[4], w[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int e = e0 + u * T;
          r[u] = 0.f; w[u] = 0.f;
          unsigned g; int i, j, k;
          if (e < nE && dense_global(a, S, S.eSelf[e], g, i, j, k)) { r[u] = __ldcg(a.rhs + g); w[u] = __ldcg(a.pw + g); }
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int e = e0 + u * T;
          if (e < nE) { S.eRhs[e] = r[u]; S.ePw[e] = w[u]; }
        }
      }
    }
    if (tid == 0 && nReload > kLMax) sOverflow = 1;
    __syncthreads();
    if (tid == 0 && sOverflow) atomicOr(&a.ctl->overflow, 1);
    // the owned cells' exchange words start with tag 0 (epochs count from 1)
    if (!sOverflow) {
      const int nOwn = bucket[0] + bucket[4];
      for (int e = tid; e < nOwn; e += T) {
        st_relaxed_u64(a.xq + S.oGlob[e], 0ull);
        st_relaxed_u64(a.xq + (size_t)d.nCells + S.oGlob[e], 0ull);
      }
    }
  }
  if (!tb_grid_barrier(a.ctl, a.err, &sAbort)) goto done;
  if (tid == 0) sOverflow = (int)ld_acquire(reinterpret_cast<const unsigned*>(&a.ctl->overflow));
  __syncthreads();

  if (sOverflow == 0) {
    // ---- phase 3: temporal-blocked iterations
    int cum[2][4];
#pragma unroll
    for (int c = 0; c < 2; c++) {
      int acc = 0;
#pragma unroll
      for (int dd = 0; dd < 4; dd++) { acc += bucket[c * 4 + dd]; cum[c][dd] = acc; }
    }
    const int st0 = bstart[0], st1 = bstart[4];
    const int nOwn0 = bucket[0], nOwn1 = bucket[4];
    const double om1 = a.om1;
    unsigned epoch = 0;
    int nChecks = 0;
    bool fresh = true, checked = false;
    // the halo values of epoch `target`: four loads in flight per thread,
    // then each word polled again (bounded) until its tag reads target
    auto wait_and_reload = [&](unsigned target) -> bool {
      const unsigned long long* src = a.xq + (size_t)(target & 1u) * (size_t)d.nCells;
      for (int l0 = tid; l0 < nReload; l0 += 4 * T) {
        unsigned long long v[4];
#pragma unroll
        for (int u = 0; u < 4; u++) { const int l = l0 + u * T; v[u] = l < nReload ? ld_relaxed_u64(src + S.lGlob[l]) : 0ull; }
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int l = l0 + u * T;
          if (l >= nReload) continue;
          long long n = 0;
          while ((unsigned)(v[u] >> 32) != target) {
            if (++n > kTbSpinLimit || *(volatile int*)&sAbort) {
              if (n > kTbSpinLimit) atomicOr(a.err, WS_DERR_TIMEOUT);
              sAbort = 1;
              break;
            }
            v[u] = ld_relaxed_u64(src + S.lGlob[l]);
          }
          S.q[S.lDense[l]] = __uint_as_float((unsigned)v[u]);
        }
      }
      __syncthreads();
      return *(volatile int*)&sAbort == 0;
    };
    // the owned cells of epoch `ep` into exchange buffer ep & 1
    auto publish_owned = [&](unsigned ep) {
      unsigned long long* dst = a.xq + (size_t)(ep & 1u) * (size_t)d.nCells;
      const unsigned long long tag = (unsigned long long)ep << 32;
      for (int e = tid; e < nOwn0 + nOwn1; e += T)
        st_relaxed_u64(dst + S.oGlob[e], tag | __float_as_uint(S.q[S.eSelf[e < nOwn0 ? st0 + e : st1 + (e - nOwn0)]]));
    };
    auto write_owned = [&](float* dst) {
      for (int e = tid; e < nOwn0 + nOwn1; e += T)
        __stcg(dst + S.oGlob[e], S.q[S.eSelf[e < nOwn0 ? st0 + e : st1 + (e - nOwn0)]]);
    };
    auto check_residual = [&]() -> bool {
      const double2 part = owned_residual(a, S, O, sRed);
      if (!global_residual(a, part, nChecks++, &sRel, &sAbort)) return false;
      rel = sRel;
      return true;
    };
    while (it < a.iters) {
      int m = std::min(2, a.iters - it);
      if (a.check > 0) m = std::min(m, a.check - it % a.check);
      if (!fresh && !wait_and_reload(epoch)) goto done;
      const int s = 2 * m;
      for (int t = 1; t <= s; t++) {
        const int col = (t - 1) & 1, dmax = s - t;
        const int n = cum[col][dmax], base = col ? st1 : st0;
        // two updates per thread in flight where a thread has two entries
        // (e and e + T are of one colour, so neither reads what the other
        // writes); a thread with one entry reads nothing extra
        for (int e = tid; e < n; e += 2 * T) {
          const int i1 = base + e, e2 = e + T;
          const unsigned a0 = S.eNb[i1][0], a1 = S.eNb[i1][1], a2 = S.eNb[i1][2];
          float v[6];
          v[0] = S.q[a0 & 0xffffu]; v[1] = S.q[a0 >> 16]; v[2] = S.q[a1 & 0xffffu];
          v[3] = S.q[a1 >> 16]; v[4] = S.q[a2 & 0xffffu]; v[5] = S.q[a2 >> 16];
          const int x1 = S.eSelf[i1];
          if (e2 < n) {
            const int i2 = base + e2;
            const unsigned b0 = S.eNb[i2][0], b1 = S.eNb[i2][1], b2 = S.eNb[i2][2];
            float u[6];
            u[0] = S.q[b0 & 0xffffu]; u[1] = S.q[b0 >> 16]; u[2] = S.q[b1 & 0xffffu];
            u[3] = S.q[b1 >> 16]; u[4] = S.q[b2 & 0xffffu]; u[5] = S.q[b2 >> 16];
            const int x2 = S.eSelf[i2];
            const float q1 = relax(S.q[x1], S.ePw[i1], S.eRhs[i1], v, om1);
            const float q2 = relax(S.q[x2], S.ePw[i2], S.eRhs[i2], u, om1);
            S.q[x1] = q1;
            S.q[x2] = q2;
          } else {
            S.q[x1] = relax(S.q[x1], S.ePw[i1], S.eRhs[i1], v, om1);
          }
        }
        __syncthreads();
      }
      it += m;
      epoch++;
      // no barrier before the reload that follows: it writes halo cells
      // (d >= 1) of S.q, this reads owned cells (d = 0)
      publish_owned(epoch);
      fresh = false;
      checked = false;
      const bool doCheck = a.check > 0 && it % a.check == 0;
      if (doCheck || it >= a.iters) {
        if (!wait_and_reload(epoch)) goto done;
        fresh = true;
        if (!check_residual()) goto done;
        checked = true;
        if (doCheck && rel <= a.tol) break;
      }
    }
    if (!checked && !check_residual()) goto done;           // no iteration ran: residual of the start
    // the result lands in the solve's own q buffer
    write_owned(a.q);
  } else {
    // ---- fallback: red-black sweeps over the owned bricks in global memory,
    // a grid barrier per half-sweep
    path = 4;
    const int t0 = sT0;
    O = sT1 - sT0;
    const double om1 = a.om1;
    const long long nxl = d.nx, nxy = (long long)d.nx * d.ny;
    int nChecks = 0;
    auto cell_of = [&](int item, int col, long long& g) -> bool {
      const int s = item >> 5, kk = item & 31, row = kk >> 1, cy = row & 3, cz = row >> 2;
      const int cx = ((col + cy + cz) & 1) + 2 * (kk & 1);
      const int lin = __ldcg(&a.actLin[t0 + s]);
      const int bx = lin % a.nbx, tq = lin / a.nbx, by = tq % a.nby, bz = tq / a.nby;
      const int i = bx * 4 + cx, j = by * 4 + cy, k = bz * 4 + cz;
      if (i >= d.nx || j >= d.ny || k >= d.nz || !interior(d, i, j, k)) return false;
      g = ((long long)k * d.ny + j) * d.nx + i;
      return __ldcg(a.pw + g) >= 0.f;
    };
    auto residual = [&]() -> bool {
      double rr = 0, bb = 0;
      for (int col = 0; col < 2; col++)
        for (int item = tid; item < O * 32; item += T) {
          long long g;
          if (!cell_of(item, col, g)) continue;
          const float* qc = a.q + g;
          double sum = (double)__ldcg(qc - 1);
          sum += (double)__ldcg(qc + 1); sum += (double)__ldcg(qc - nxl); sum += (double)__ldcg(qc + nxl);
          sum += (double)__ldcg(qc - nxy); sum += (double)__ldcg(qc + nxy);
          const double b = a.rhs[g];
          const double r = b + sum - (double)a.diag8[g] * (double)__ldcg(qc);
          rr += r * r; bb += b * b;
        }
      rr = warp_sum(rr); bb = warp_sum(bb);
      if (lane == 0) sRed[tid >> 5] = make_double2(rr, bb);
      __syncthreads();
      double2 part = make_double2(0, 0);
      if (tid < 32) {
        const double2 v = tid < (T >> 5) ? sRed[tid] : make_double2(0, 0);
        part = make_double2(warp_sum(v.x), warp_sum(v.y));
      }
      __syncthreads();
      if (!global_residual(a, part, nChecks++, &sRel, &sAbort)) return false;
      rel = sRel;
      return true;
    };
    bool checked = false;
    while (it < a.iters) {
      for (int col = 0; col < 2; col++) {
        for (int item = tid; item < O * 32; item += T) {
          long long g;
          if (!cell_of(item, col, g)) continue;
          float* qc = a.q + g;
          float v[6];
          v[0] = __ldcg(qc - 1); v[1] = __ldcg(qc + 1); v[2] = __ldcg(qc - nxl);
          v[3] = __ldcg(qc + nxl); v[4] = __ldcg(qc - nxy); v[5] = __ldcg(qc + nxy);
          __stcg(qc, relax(__ldcg(qc), a.pw[g], a.rhs[g], v, om1));
        }
        if (!tb_grid_barrier(a.ctl, a.err, &sAbort)) goto done;
      }
      it++;
      checked = false;
      const bool doCheck = a.check > 0 && it % a.check == 0;
      if (doCheck) {
        if (!residual()) goto done;
        checked = true;
        if (rel <= a.tol) break;
      }
    }
    if (!checked && !residual()) goto done;
  }
done:
  if (p == 0 && tid == 0) { *a.outIters = it; *a.outRel = rel; *a.outPath = path; }
}

// ---------------------------------------------------------------- host side
struct TbState {
  TbCtl* ctl = nullptr;
  unsigned long long* xq = nullptr;
  int* brickW = nullptr;
  int2* cntPart = nullptr;
  int *actLin = nullptr, *actWPre = nullptr, *brickOrd = nullptr, *chunkStart = nullptr;
  double2* resPart = nullptr;
  int P = 0, nbx = 0, nby = 0, nbz = 0, mbits = 0;
};

size_t sor_tb_smem_bytes() { return sizeof(TbSmem); }

// 0 when the temporal-blocked solve cannot run on this device (too little
// shared memory or co-residency); the state is then left unallocated.
cudaError_t sor_tb_init(void** statePtr, const Dims& d, int device) {
  *statePtr = nullptr;
  int smCount = 0, optin = 0;
  cudaDeviceGetAttribute(&smCount, cudaDevAttrMultiProcessorCount, device);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  if (smCount < 1 || smCount > kMaxCtas || optin < (int)sizeof(TbSmem)) return cudaSuccess;
  if (cudaFuncSetAttribute(k_sor_tb, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TbSmem)) != cudaSuccess) {
    cudaGetLastError();
    return cudaSuccess;
  }
  int perSM = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k_sor_tb, kTbThreads, sizeof(TbSmem)) != cudaSuccess ||
      perSM < 1) {
    cudaGetLastError();
    return cudaSuccess;
  }
  TbState* S = new TbState();
  S->P = smCount;
  S->nbx = (d.nx + 3) / 4; S->nby = (d.ny + 3) / 4; S->nbz = (d.nz + 3) / 4;
  int mb = 0;
  while ((1 << mb) < std::max(S->nbx, std::max(S->nby, S->nbz))) mb++;
  S->mbits = mb;
  const long long nB = (long long)S->nbx * S->nby * S->nbz, MC = 1LL << (3 * mb);
  cudaError_t e;
  if ((e = cudaMalloc(&S->ctl, sizeof(TbCtl))) != cudaSuccess) return e;
  if ((e = cudaMalloc(&S->xq, sizeof(unsigned long long) * 2 * d.nCells)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&S->brickW, sizeof(int) * MC)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&S->cntPart, sizeof(int2) * smCount)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&S->actLin, sizeof(int) * nB)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&S->actWPre, sizeof(int) * nB)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&S->brickOrd, sizeof(int) * nB)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&S->chunkStart, sizeof(int) * (smCount + 1))) != cudaSuccess) return e;
  if ((e = cudaMalloc(&S->resPart, sizeof(double2) * 2 * smCount)) != cudaSuccess) return e;
  *statePtr = S;
  return cudaSuccess;
}

void sor_tb_free(void* statePtr) {
  TbState* S = (TbState*)statePtr;
  if (!S) return;
  cudaFree(S->ctl); cudaFree(S->xq); cudaFree(S->brickW); cudaFree(S->cntPart); cudaFree(S->actLin);
  cudaFree(S->actWPre); cudaFree(S->brickOrd); cudaFree(S->chunkStart); cudaFree(S->resPart);
  delete S;
}

// the control block reset and the solve (two stream operations, one kernel)
cudaError_t launch_sor_tb(void* statePtr, const Dims& d, const GridDev& g, const uint8_t* diag8, double omega,
                          int iters, int check, double tol, int* err, int* outIters, double* outRel, int* outPath,
                          cudaStream_t s) {
  TbState* S = (TbState*)statePtr;
  cudaError_t e = cudaMemsetAsync(S->ctl, 0, sizeof(TbCtl), s);
  if (e != cudaSuccess) return e;
  TbArgs a;
  a.d = d; a.q = g.q; a.xq = S->xq; a.rhs = g.rhs; a.pw = g.pw; a.diag8 = diag8;
  a.nbx = S->nbx; a.nby = S->nby; a.nbz = S->nbz; a.mbits = S->mbits;
  a.brickW = S->brickW; a.cntPart = S->cntPart; a.actLin = S->actLin; a.actWPre = S->actWPre;
  a.brickOrd = S->brickOrd; a.chunkStart = S->chunkStart; a.resPart = S->resPart; a.ctl = S->ctl;
  a.om1 = 1 - omega; a.iters = iters; a.check = check; a.tol = tol; a.err = err;
  a.outIters = outIters; a.outRel = outRel; a.outPath = outPath;
  void* args[] = { &a };
  return cudaLaunchCooperativeKernel((void*)k_sor_tb, dim3(S->P), dim3(kTbThreads), args, sizeof(TbSmem), s);
}
