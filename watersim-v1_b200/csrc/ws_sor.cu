// ws_sor.cu — the pressure solve of _pressureSolve (js/solver.js:1368-1404)
// as one persistent cooperative kernel.
//
// The fluid cells (about 5% of the 128^3 box) are compacted per red-black
// colour into lists in cell order (rhs, omega/diag and diag copied beside
// each index). One kernel then runs every sweep of the solve: each block
// strides over the colour lists, and a software grid barrier separates the
// half-sweeps, so no launch and no host round trip sits between them. The
// FP64 residual check (||b - A q|| / ||b||, every sorCheckEvery iterations)
// is reduced in the kernel: block partials are summed in block order by
// every block, so all blocks take the same stop decision and the value is
// deterministic. q neighbours are read with ld.global.cg (L2) because other
// SMs wrote them in the previous half-sweep.
//
// Every barrier wait is bounded: after kSpinLimit polls the block latches
// WS_DERR_TIMEOUT in the status word and the solve ends early; the host
// reports WS_ERR_TIMEOUT. The cooperative launch guarantees co-residency,
// so a healthy run never reaches the limit.
#include "ws_kernels.cuh"
#include <algorithm>
#include <cooperative_groups.h>

static const long long kSpinLimit = 4000000LL;

struct SorLists {
  int* idx[2];
  float* rhs[2];
  float* pw[2];
  uint8_t* dg[2];
  uint16_t* code[2];   // 6 neighbour codes per entry for the cluster solve
  int* pos;            // dense: list position of each listed cell
  int* count;          // [2] list lengths (device)
};

// Cluster-resident solve: one cluster of kClusterMax CTAs holds every fluid
// cell. A CTA owns at most kSmax cells per colour; a neighbour code packs the
// owner's rank (4 bits) and slot (12 bits); slot kSmax is a zero (non-fluid).
#define kClusterMax 16
#define kSmax 4095

// ---------------------------------------------------------------- list build
// colour of an interior fluid cell (pw >= 0 marks fluid), -1 otherwise; fluid
// never touches the solid domain shell, and the interior test keeps every
// stencil read inside the grid whatever state a caller uploads
__device__ __forceinline__ int sor_colour(const Dims& d, const float* __restrict__ pw, unsigned c) {
  if (c >= (unsigned)d.nCells || pw[c] < 0.f) return -1;
  unsigned nx = d.nx, ny = d.ny;
  unsigned t = fastdiv(c, d.dnx), i = c - t * nx, k = fastdiv(t, d.dny), j = t - k * ny;
  if (i < 1 || j < 1 || k < 1 || i + 2 > nx || j + 2 > ny || (int)k + 2 > d.nz) return -1;
  return (int)((i + j + k) & 1u);
}
// exclusive scan of the (colour 0, colour 1) block counts into offs, one
// block of 32 warps: each warp owns a contiguous segment and reads it 32 pairs
// at a time (coalesced); pass 1 sums the segments, the block scans the 32
// sums, pass 2 rescans each segment from its carry and writes the offsets.
// total = the two list lengths. The counts stay as the pressure setup wrote
// them, so the solve can be repeated on the same system.
__global__ void __launch_bounds__(1024) k_sor_scan(const int* __restrict__ blockCounts, int nb, int* __restrict__ offs,
                                                   int* __restrict__ total) {
  __shared__ int w0[32], w1[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int2* cnt = reinterpret_cast<const int2*>(blockCounts);
  int2* out = reinterpret_cast<int2*>(offs);
  const int seg = (nb + nw - 1) / nw, lo = min(nb, wid * seg), hi = min(nb, lo + seg);
  int s0 = 0, s1 = 0;
  for (int i = lo + lane; i < hi; i += 32) { int2 v = cnt[i]; s0 += v.x; s1 += v.y; }
  s0 = __reduce_add_sync(0xffffffffu, s0); s1 = __reduce_add_sync(0xffffffffu, s1);
  if (lane == 0) { w0[wid] = s0; w1[wid] = s1; }
  __syncthreads();
  if (wid == 0) {
    int a = lane < nw ? w0[lane] : 0, b = lane < nw ? w1[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      int ya = __shfl_up_sync(0xffffffffu, a, o), yb = __shfl_up_sync(0xffffffffu, b, o);
      if (lane >= o) { a += ya; b += yb; }
    }
    w0[lane] = a; w1[lane] = b;
  }
  __syncthreads();
  int c0 = wid > 0 ? w0[wid - 1] : 0, c1 = wid > 0 ? w1[wid - 1] : 0;   // this segment's carry
  for (int base = lo; base < hi; base += 32) {
    const int i = base + lane;
    int2 v = i < hi ? cnt[i] : make_int2(0, 0);
    int x0 = v.x, x1 = v.y;
    for (int o = 1; o < 32; o <<= 1) {
      int y0 = __shfl_up_sync(0xffffffffu, x0, o), y1 = __shfl_up_sync(0xffffffffu, x1, o);
      if (lane >= o) { x0 += y0; x1 += y1; }
    }
    if (i < hi) out[i] = make_int2(c0 + x0 - v.x, c1 + x1 - v.y);
    c0 += __shfl_sync(0xffffffffu, x0, 31); c1 += __shfl_sync(0xffffffffu, x1, 31);
  }
  if (threadIdx.x == 0) { total[0] = w0[nw - 1]; total[1] = w1[nw - 1]; }
}
// Persistent over the 256-cell chunks the pressure setup counted (chunk b
// holds cells 256 b .. 256 b + 255 and its list offsets are offs[2 b], offs[2 b
// + 1]); the next chunk's colours and offsets are fetched before this chunk's
// ranks are formed. Warp totals are double-buffered: one barrier per chunk.
__global__ void __launch_bounds__(256) k_sor_scatter(Dims d, const float* __restrict__ pw, const float* __restrict__ rhs,
                                                     const uint8_t* __restrict__ diag8, const int* __restrict__ offs,
                                                     SorLists L, int nChunks) {
  __shared__ int wt[2][2][8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int b = blockIdx.x;
  unsigned c = (unsigned)b * 256u + threadIdx.x;
  int col = b < nChunks ? sor_colour(d, pw, c) : -1;
  int o0 = b < nChunks ? offs[2 * b] : 0, o1 = b < nChunks ? offs[2 * b + 1] : 0;
  int buf = 0;
  for (; b < nChunks; b += gridDim.x) {
    const int bn = b + (int)gridDim.x;
    const unsigned cn = (unsigned)bn * 256u + threadIdx.x;
    const int coln = bn < nChunks ? sor_colour(d, pw, cn) : -1;
    const int o0n = bn < nChunks ? offs[2 * bn] : 0, o1n = bn < nChunks ? offs[2 * bn + 1] : 0;
    const unsigned m0 = __ballot_sync(0xffffffffu, col == 0), m1 = __ballot_sync(0xffffffffu, col == 1);
    if (lane == 0) { wt[buf][0][wid] = __popc(m0); wt[buf][1][wid] = __popc(m1); }
    __syncthreads();
    if (col >= 0) {
      const unsigned m = col ? m1 : m0;
      int e = (col ? o1 : o0) + __popc(m & ((1u << lane) - 1u));
      for (int w = 0; w < wid; w++) e += wt[buf][col][w];
      (col ? L.idx[1] : L.idx[0])[e] = (int)c;      // selects, not a dynamic index into the parameter
      (col ? L.rhs[1] : L.rhs[0])[e] = rhs[c];
      (col ? L.pw[1] : L.pw[0])[e] = pw[c];
      (col ? L.dg[1] : L.dg[0])[e] = diag8[c];
      L.pos[c] = e;
    }
    c = cn; col = coln; o0 = o0n; o1 = o1n; buf ^= 1;
  }
}
// neighbour codes (-x, +x, -y, +y, -z, +z) for the cluster solve: the owner
// rank and slot of each fluid neighbour (always of the other colour); one
// thread per (list entry, direction), so the six lookups of a cell run in
// parallel
__global__ void k_sor_codes(Dims d, const float* __restrict__ pw, SorLists L, int C) {
  const int col = blockIdx.y;
  const int n = L.count[col], nOther = L.count[1 - col];
  if (n > C * kSmax || nOther > C * kSmax) return;
  const int S = (nOther + C - 1) / C, Sown = (n + C - 1) / C;
  const long long nx = d.nx, nxy = (long long)d.nx * d.ny;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const int* __restrict__ idx = col ? L.idx[1] : L.idx[0];   // selects, not a dynamic index into the parameter
  uint16_t* __restrict__ codes = col ? L.code[1] : L.code[0];
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 6LL * n; t += stride) {
    const int e = (int)(t / 6), q = (int)(t - (long long)e * 6);
    const long long c = idx[e];
    const long long nb = c + (q == 0 ? -1 : q == 1 ? 1 : q == 2 ? -nx : q == 3 ? nx : q == 4 ? -nxy : nxy);
    // a non-fluid neighbour reads the owner CTA's own zero slot (no remote traffic)
    uint16_t code = (uint16_t)(((e / Sown) << 12) | kSmax);
    if (sor_colour(d, pw, (unsigned)nb) >= 0) {
      const int e2 = L.pos[nb];
      const int r = e2 / S, slot = e2 - r * S;
      code = (uint16_t)((r << 12) | slot);
    }
    codes[t] = code;
  }
}

// ---------------------------------------------------------------- grid barrier
// grid barrier counters, then (own cache lines) one half-sweep counter per CTA
constexpr int kMaxSorCtas = 1024;
struct GridBar { unsigned count; unsigned gen; unsigned pad[30]; unsigned flag[kMaxSorCtas]; };

__device__ __forceinline__ bool grid_barrier(GridBar* bar, unsigned nblocks, int* err) {
  __syncthreads();
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    volatile unsigned* vgen = &bar->gen;
    unsigned g = *vgen;
    __threadfence();
    int ok = 1;
    if (atomicAdd(&bar->count, 1u) == nblocks - 1) {
      atomicExch(&bar->count, 0u);
      __threadfence();
      atomicAdd(&bar->gen, 1u);
    } else {
      long long n = 0;
      while (*vgen == g) {
        if (++n > kSpinLimit) { atomicOr(err, WS_DERR_TIMEOUT); ok = 0; break; }
      }
    }
    __threadfence();
    if (*(volatile int*)err & WS_DERR_TIMEOUT) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// ---------------------------------------------------------------- solve
struct SorArgs {
  Dims d;
  float* q;
  SorLists L;
  double om1;
  int iters;           // fixed iteration count, or the cap in tolerance mode
  int check;           // residual cadence in tolerance mode (0: fixed mode)
  double tol;
  GridBar* bar;
  double2* partials;   // gridDim.x
  int* err;            // DevStatus::err
  int* outIters;
  double* outRel;
  int* outPath;
  int clusterCap;      // lists up to this size per colour were solved by k_sor_cluster
  const int* offs;     // per 256-cell chunk b: its first list entry of colour 0 and 1 (offs[2 b], offs[2 b + 1])
  int nChunks;
};

// One colour's half-sweep over the lists in global memory, three cells per
// thread at a time: every load of the three (list entry, six neighbours, own q)
// is issued before any store, so a thread pays one list round trip and one q
// round trip per batch instead of per cell. Cells of one colour never
// neighbour each other, so the batch reads no value it writes.
constexpr int kSorBatch = 3;
__device__ __forceinline__ void sor_half(const SorArgs& a, int col, unsigned lo, unsigned hi) {
  const unsigned n = hi, tid = lo + threadIdx.x, T = blockDim.x;
  const int* __restrict__ idx = a.L.idx[col];
  const float* __restrict__ rhs = a.L.rhs[col];
  const float* __restrict__ pw = a.L.pw[col];
  float* q = a.q;
  const int nx = a.d.nx, nxy = a.d.nx * a.d.ny;              // cell indices fit in 32 bits (list entries are int)
  for (unsigned e0 = tid; e0 < n; e0 += kSorBatch * T) {
    int c[kSorBatch];
    float r[kSorBatch], w[kSorBatch], v[kSorBatch][7];
#pragma unroll
    for (int j = 0; j < kSorBatch; j++) {
      const unsigned e = e0 + j * T;
      c[j] = e < n ? idx[e] : -1;
      r[j] = e < n ? rhs[e] : 0.f;
      w[j] = e < n ? pw[e] : 0.f;
    }
#pragma unroll
    for (int j = 0; j < kSorBatch; j++) {
      if (c[j] < 0) continue;
      const float* qc = q + c[j];
      v[j][0] = __ldcg(qc - 1); v[j][1] = __ldcg(qc + 1); v[j][2] = __ldcg(qc - nx); v[j][3] = __ldcg(qc + nx);
      v[j][4] = __ldcg(qc - nxy); v[j][5] = __ldcg(qc + nxy); v[j][6] = __ldcg(qc);
    }
#pragma unroll
    for (int j = 0; j < kSorBatch; j++) {
      if (c[j] < 0) continue;
      __stcg(q + c[j], sor_update(v[j][6], w[j], r[j], v[j][0], v[j][1], v[j][2], v[j][3], v[j][4], v[j][5],
                                  a.om1));
    }
  }
}

// residual partial of this block (both colours) -> partials[blockIdx.x]
__device__ void residual_block(const SorArgs& a, unsigned tid, unsigned T) {
  __shared__ double srr[32], sbb[32];
  double rr = 0, bb = 0;
  const long long nx = a.d.nx, nxy = (long long)a.d.nx * a.d.ny;
  const float* q = a.q;
  for (int col = 0; col < 2; col++) {
    const int n = a.L.count[col];
    for (unsigned e = tid; e < (unsigned)n; e += T) {
      long long c = a.L.idx[col][e];
      double sum = (double)__ldcg(q + c - 1);
      sum += (double)__ldcg(q + c + 1); sum += (double)__ldcg(q + c - nx); sum += (double)__ldcg(q + c + nx);
      sum += (double)__ldcg(q + c - nxy); sum += (double)__ldcg(q + c + nxy);
      double b = a.L.rhs[col][e];
      double r = b + sum - (double)a.L.dg[col][e] * (double)__ldcg(q + c);
      rr += r * r; bb += b * b;
    }
  }
  rr = warp_sum(rr); bb = warp_sum(bb);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { srr[wid] = rr; sbb[wid] = bb; }
  __syncthreads();
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    rr = lane < nw ? srr[lane] : 0; bb = lane < nw ? sbb[lane] : 0;
    rr = warp_sum(rr); bb = warp_sum(bb);
    if (lane == 0) __stcg(&a.partials[blockIdx.x], make_double2(rr, bb));
  }
}
// every block sums the partials in block order: identical value everywhere
__device__ double residual_total(const SorArgs& a) {
  __shared__ double s_rel;
  if (threadIdx.x < 32) {
    double rr = 0, bb = 0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += 32) { double2 p = __ldcg(&a.partials[b]); rr += p.x; bb += p.y; }
    rr = warp_sum(rr); bb = warp_sum(bb);
    if (threadIdx.x == 0) s_rel = bb > 0 ? sqrt(rr) / sqrt(bb) : sqrt(rr);
  }
  __syncthreads();
  return s_rel;
}

// One list entry held in registers for the whole solve: cell index, rhs,
// omega/diag, diag and the cell's own q (only its owner thread writes it).
struct Entry { long long c; float rhs, pw, q; uint8_t dg; };

__device__ __forceinline__ void entry_relax(Entry& e, const float* q, long long nx, long long nxy, double om1) {
  if (e.c < 0) return;
  const float n0 = __ldcg(q + e.c - 1), n1 = __ldcg(q + e.c + 1), n2 = __ldcg(q + e.c - nx);
  const float n3 = __ldcg(q + e.c + nx), n4 = __ldcg(q + e.c - nxy), n5 = __ldcg(q + e.c + nxy);
  e.q = sor_update(e.q, e.pw, e.rhs, n0, n1, n2, n3, n4, n5, om1);
  __stcg(const_cast<float*>(q) + e.c, e.q);
}
__device__ __forceinline__ void entry_residual(const Entry& e, const float* q, long long nx, long long nxy,
                                               double& rr, double& bb) {
  if (e.c < 0) return;
  double sum = (double)__ldcg(q + e.c - 1);
  sum += (double)__ldcg(q + e.c + 1); sum += (double)__ldcg(q + e.c - nx); sum += (double)__ldcg(q + e.c + nx);
  sum += (double)__ldcg(q + e.c - nxy); sum += (double)__ldcg(q + e.c + nxy);
  double b = e.rhs;
  double r = b + sum - (double)e.dg * (double)e.q;
  rr += r * r; bb += b * b;
}
__device__ __forceinline__ void block_partial(const SorArgs& a, double rr, double bb) {
  __shared__ double srr[32], sbb[32];
  rr = warp_sum(rr); bb = warp_sum(bb);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { srr[wid] = rr; sbb[wid] = bb; }
  __syncthreads();
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    rr = lane < nw ? srr[lane] : 0; bb = lane < nw ? sbb[lane] : 0;
    rr = warp_sum(rr); bb = warp_sum(bb);
    if (lane == 0) __stcg(&a.partials[blockIdx.x], make_double2(rr, bb));
  }
}

// release / acquire of the per-CTA half-sweep counters
__device__ __forceinline__ void sor_publish(unsigned* flag, unsigned v) {
  asm volatile("fence.acq_rel.gpu;" ::: "memory");
  asm volatile("st.release.gpu.global.u32 [%0], %1;" :: "l"(flag), "r"(v) : "memory");
}

// The iteration loop, in two instantiations so that the register-resident
// entries of the cached path are not live in the list-reading path.
//
// Cached path (each thread holds at most one cell per colour): a grid
// barrier after every half-sweep. List path: CTA p sweeps the contiguous
// range [ceil(p n / P), ceil((p + 1) n / P)) of each colour list (cells in
// cell order, so a compact run of z-planes), and a half-sweep waits only for
// the CTAs owning other-colour cells within one z-plane (nx ny cells) of its
// range: those it reads, and those that read the cells it writes. Each CTA
// publishes its count of finished half-sweeps (release) and polls its
// neighbours' (acquire, bounded); the residual checks keep grid barriers.
template <bool CACHED>
__device__ __forceinline__ void persistent_loop(const SorArgs& a, unsigned tid, unsigned T) {
  const int n0 = a.L.count[0], n1 = a.L.count[1];
  const long long nx = a.d.nx, nxy = (long long)a.d.nx * a.d.ny;
  __shared__ int sLo[2], sHi[2], sDl[2], sDh[2], sAbort;
  Entry e0, e1;
  e0.c = -1; e1.c = -1;
  if (CACHED) {
    if (tid < (unsigned)n0) { e0.c = a.L.idx[0][tid]; e0.rhs = a.L.rhs[0][tid]; e0.pw = a.L.pw[0][tid]; e0.dg = a.L.dg[0][tid]; e0.q = __ldcg(a.q + e0.c); }
    if (tid < (unsigned)n1) { e1.c = a.L.idx[1][tid]; e1.rhs = a.L.rhs[1][tid]; e1.pw = a.L.pw[1][tid]; e1.dg = a.L.dg[1][tid]; e1.q = __ldcg(a.q + e1.c); }
  } else {
    if (threadIdx.x == 0) {
      const long long P = gridDim.x, p = blockIdx.x;
      sAbort = 0;
      for (int c = 0; c < 2; c++) {
        const long long n = c ? n1 : n0, no = c ? n0 : n1;
        const int lo = (int)((p * n + P - 1) / P), hi = (int)(((p + 1) * n + P - 1) / P);
        sLo[c] = lo; sHi[c] = hi;
        int dl = (int)p, dh = (int)p;
        if (hi > lo && no > 0) {
          const long long cLo = (long long)(c ? a.L.idx[1] : a.L.idx[0])[lo] - nxy;
          const long long cHi = (long long)(c ? a.L.idx[1] : a.L.idx[0])[hi - 1] + nxy;
          const int bLo = cLo < 0 ? 0 : (int)(cLo / 256);
          const int bHi = (int)std::min<long long>(a.nChunks - 1, cHi / 256);
          const long long eLo = a.offs[2 * bLo + (1 - c)];
          const long long eHi = bHi + 1 < a.nChunks ? a.offs[2 * (bHi + 1) + (1 - c)] : no;   // exclusive
          if (eHi > eLo) { dl = (int)(eLo * P / no); dh = (int)((eHi - 1) * P / no); }
        }
        sDl[c] = dl; sDh[c] = dh;
      }
    }
    __syncthreads();
  }
  auto partial = [&]() {
    if (CACHED) { double rr = 0, bb = 0; entry_residual(e0, a.q, nx, nxy, rr, bb); entry_residual(e1, a.q, nx, nxy, rr, bb); block_partial(a, rr, bb); }
    else residual_block(a, tid, T);
  };
  // list path: before a half-sweep of colour c, the neighbours of that colour
  // have finished `done` half-sweeps
  auto wait_deps = [&](int c, unsigned done) -> bool {
    if (threadIdx.x < 32) {
      for (int q = sDl[c] + (int)threadIdx.x; q <= sDh[c]; q += 32)
        if (q != (int)blockIdx.x && !bounded_wait_geq(&a.bar->flag[q], done, kSpinLimit, a.err)) sAbort = 1;
    }
    __syncthreads();
    return *(volatile int*)&sAbort == 0;
  };
  auto finish_half = [&](unsigned done) {
    __syncthreads();                       // every thread's stores before thread 0's release
    if (threadIdx.x == 0) sor_publish(&a.bar->flag[blockIdx.x], done);
  };
  int it = 0;
  bool ok = true;
  double rel = -1;
  unsigned done = 0;
  for (it = 0; it < a.iters && ok; ) {
    if (CACHED) {
      entry_relax(e0, a.q, nx, nxy, a.om1);
      if (!(ok = grid_barrier(a.bar, gridDim.x, a.err))) break;
      entry_relax(e1, a.q, nx, nxy, a.om1);
      if (!(ok = grid_barrier(a.bar, gridDim.x, a.err))) break;
    } else {
      if (done > 0 && !(ok = wait_deps(0, done))) break;
      sor_half(a, 0, (unsigned)sLo[0], (unsigned)sHi[0]);
      finish_half(++done);
      if (!(ok = wait_deps(1, done))) break;
      sor_half(a, 1, (unsigned)sLo[1], (unsigned)sHi[1]);
      finish_half(++done);
    }
    it++;
    if (a.check > 0 && it % a.check == 0) {
      if (!CACHED && !(ok = grid_barrier(a.bar, gridDim.x, a.err))) break;   // every half-sweep finished
      partial();
      if (!(ok = grid_barrier(a.bar, gridDim.x, a.err))) break;
      rel = residual_total(a);
      if (!(ok = grid_barrier(a.bar, gridDim.x, a.err))) break;   // partials reusable
      if (rel <= a.tol) break;
    }
  }
  if (ok) {
    if (!CACHED) ok = grid_barrier(a.bar, gridDim.x, a.err);
    if (ok) partial();
    if (ok) ok = grid_barrier(a.bar, gridDim.x, a.err);
    if (ok) rel = residual_total(a);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) { *a.outIters = it; *a.outRel = rel; *a.outPath = 1; }
}
__global__ void __launch_bounds__(1024, 1) k_sor_persistent(SorArgs a) {
  const unsigned T = gridDim.x * blockDim.x;
  const unsigned tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int n0 = a.L.count[0], n1 = a.L.count[1];
  if (n0 <= a.clusterCap && n1 <= a.clusterCap) return;      // the cluster solve ran
  if (n0 + n1 == 0) {                  // no fluid cell: no sweep (js/solver.js:1330)
    if (tid == 0) { *a.outIters = 0; *a.outRel = 0; *a.outPath = 1; }
    return;
  }
  // register-resident path when every thread owns at most one cell per colour
  if ((unsigned)n0 <= T && (unsigned)n1 <= T) persistent_loop<true>(a, tid, T);
  else persistent_loop<false>(a, tid, T);
}


// ---------------------------------------------------------------- cluster solve
// The whole solve inside one thread-block cluster: each CTA keeps its share
// of the fluid cells (q, rhs, omega/diag, diag, neighbour codes) in shared
// memory, reads neighbour q from the other CTAs through distributed shared
// memory, and separates half-sweeps with the hardware cluster barrier.
// Same per-cell arithmetic and order as the reference's sweep
// (js/solver.js:1397-1404, red-black order), so results match
// k_sor_persistent bit for bit.
struct ClusterArgs {
  Dims d;
  float* q;
  SorLists L;
  double om1;
  int iters, check;
  double tol;
  int* outIters;
  double* outRel;
  int* outPath;
};
extern __shared__ __align__(16) unsigned char sor_smem[];

// Non-fluid neighbours are coded to slot kSmax of the owner CTA's own table,
// which holds 0.0f: all six loads of a cell are unconditional and
// independent, and adding +0.0 leaves the sum of the fluid neighbours
// unchanged (the reference adds only fluid neighbours).
__device__ __forceinline__ float cl_load(float* const* rq, uint16_t code) {
  return rq[code >> 12][code & 4095u];
}
// relax (or measure) up to two cells per call with all twelve loads in flight
__device__ __forceinline__ void cl_vals(const uint16_t* cd, float* const* rq, int e0, int e1, int m, float (&v)[2][6]) {
#pragma unroll
  for (int q = 0; q < 6; q++) {
    v[0][q] = e0 < m ? cl_load(rq, cd[6 * e0 + q]) : 0.f;
    v[1][q] = e1 < m ? cl_load(rq, cd[6 * e1 + q]) : 0.f;
  }
}
// FP64 sums of the six neighbours (the residual)
__device__ __forceinline__ void cl_sums(const uint16_t* cd, float* const* rq, int e0, int e1, int m,
                                        double& s0, double& s1) {
  float v[2][6];
  cl_vals(cd, rq, e0, e1, m, v);
  s0 = (double)v[0][0]; s1 = (double)v[1][0];
#pragma unroll
  for (int q = 1; q < 6; q++) { s0 += (double)v[0][q]; s1 += (double)v[1][q]; }
}

__global__ void __launch_bounds__(1024, 1) k_sor_cluster(ClusterArgs a) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const int C = (int)cl.num_blocks();
  const int rank = (int)cl.block_rank();
  const int n0 = a.L.count[0], n1 = a.L.count[1];
  if (n0 > C * kSmax || n1 > C * kSmax) return;         // uniform: the grid solve takes it
  if (n0 + n1 == 0) {                                    // no fluid cell: no sweep (js/solver.js:1330)
    if (rank == 0 && threadIdx.x == 0) { *a.outIters = 0; *a.outRel = 0; *a.outPath = 2; }
    return;
  }
  const int S0 = (n0 + C - 1) / C, S1 = (n1 + C - 1) / C;
  const int QS = kSmax + 1;                              // slot kSmax holds 0.0f
  float* qs[2]; float* rh[2]; float* pw[2]; uint16_t* cd[2]; uint8_t* dg[2];
  qs[0] = (float*)sor_smem; qs[1] = qs[0] + QS;
  rh[0] = qs[1] + QS; rh[1] = rh[0] + kSmax;
  pw[0] = rh[1] + kSmax; pw[1] = pw[0] + kSmax;
  cd[0] = (uint16_t*)(pw[1] + kSmax); cd[1] = cd[0] + 6 * kSmax;
  dg[0] = (uint8_t*)(cd[1] + 6 * kSmax); dg[1] = dg[0] + kSmax;
  __shared__ float* rq[2][kClusterMax];
  __shared__ double2 mypart;
  __shared__ double srr[32], sbb[32];
  __shared__ double s_rel;
  const int base[2] = { rank * S0, rank * S1 };
  const int m[2] = { max(0, min(S0, n0 - base[0])), max(0, min(S1, n1 - base[1])) };
  for (int col = 0; col < 2; col++) {
    for (int e = threadIdx.x; e < m[col]; e += blockDim.x) {
      int g = base[col] + e;
      qs[col][e] = __ldcg(a.q + a.L.idx[col][g]);
      rh[col][e] = a.L.rhs[col][g]; pw[col][e] = a.L.pw[col][g]; dg[col][e] = a.L.dg[col][g];
#pragma unroll
      for (int q = 0; q < 6; q++) cd[col][6 * e + q] = a.L.code[col][6 * (long long)g + q];
    }
  }
  if (threadIdx.x == 0) { qs[0][kSmax] = 0.f; qs[1][kSmax] = 0.f; }
  if (threadIdx.x < kClusterMax) {
    int r = (int)threadIdx.x;
    // own rank: plain shared-memory pointer; other ranks: the distributed-shared-memory window
    rq[0][r] = (r < C && r != rank) ? cl.map_shared_rank(qs[0], r) : qs[0];
    rq[1][r] = (r < C && r != rank) ? cl.map_shared_rank(qs[1], r) : qs[1];
  }
  cl.sync();
  const double om1 = a.om1;
  const int B = blockDim.x;
  auto residual = [&]() -> double {
    double rr = 0, bb = 0;
    for (int col = 0; col < 2; col++)
      for (int e = threadIdx.x; e < m[col]; e += 2 * B) {
        int e1 = e + B;
        double s0, s1;
        cl_sums(cd[col], rq[1 - col], e, e1, m[col], s0, s1);
        double b = rh[col][e];
        double r = b + s0 - (double)dg[col][e] * (double)qs[col][e];
        rr += r * r; bb += b * b;
        if (e1 < m[col]) {
          b = rh[col][e1];
          r = b + s1 - (double)dg[col][e1] * (double)qs[col][e1];
          rr += r * r; bb += b * b;
        }
      }
    rr = warp_sum(rr); bb = warp_sum(bb);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { srr[wid] = rr; sbb[wid] = bb; }
    __syncthreads();
    if (threadIdx.x < 32) {
      rr = lane < (int)(blockDim.x >> 5) ? srr[lane] : 0; bb = lane < (int)(blockDim.x >> 5) ? sbb[lane] : 0;
      rr = warp_sum(rr); bb = warp_sum(bb);
      if (lane == 0) mypart = make_double2(rr, bb);
    }
    cl.sync();                                               // every CTA's partial is in place
    if (threadIdx.x == 0) {
      double R = 0, Bb = 0;
      for (int r = 0; r < C; r++) { double2 p = *cl.map_shared_rank(&mypart, r); R += p.x; Bb += p.y; }
      s_rel = Bb > 0 ? sqrt(R) / sqrt(Bb) : sqrt(R);
    }
    cl.sync();                                               // partials may be rewritten after this
    return s_rel;
  };
  int it = 0;
  double rel = -1;
  for (it = 0; it < a.iters; ) {
    for (int col = 0; col < 2; col++) {
      for (int e = threadIdx.x; e < m[col]; e += 2 * B) {
        int e1 = e + B;
        float v[2][6];
        cl_vals(cd[col], rq[1 - col], e, e1, m[col], v);
        qs[col][e] = sor_update(qs[col][e], pw[col][e], rh[col][e], v[0][0], v[0][1], v[0][2], v[0][3], v[0][4],
                                v[0][5], om1);
        if (e1 < m[col])
          qs[col][e1] = sor_update(qs[col][e1], pw[col][e1], rh[col][e1], v[1][0], v[1][1], v[1][2], v[1][3],
                                   v[1][4], v[1][5], om1);
      }
      cl.sync();
    }
    it++;
    if (a.check > 0 && it % a.check == 0) {
      rel = residual();
      if (rel <= a.tol) break;
    }
  }
  rel = residual();
  for (int col = 0; col < 2; col++)
    for (int e = threadIdx.x; e < m[col]; e += blockDim.x) a.q[a.L.idx[col][base[col] + e]] = qs[col][e];
  if (rank == 0 && threadIdx.x == 0) { *a.outIters = it; *a.outRel = rel; *a.outPath = 2; }
}
static size_t cluster_smem_bytes() { return (size_t)(kSmax + 1) * 2 * 4 + (size_t)kSmax * (2 * 4 * 2 + 2 * 6 * 2 + 2); }

// ---------------------------------------------------------------- host side
struct SorState {
  SorLists L{};
  int* blockCounts = nullptr;  // per 256-cell block: interior fluid cells of colour 0, 1 (pressure setup)
  int* blockOffs = nullptr;    // their exclusive scan: each block's first list slot per colour
  GridBar* bar = nullptr;
  double2* partials = nullptr;
  int* outIters = nullptr;
  double* outRel = nullptr;
  int* outPath = nullptr;
  int grid = 0, block = 1024;
  long long cap = 0;
  int clusterSize = 0;       // 0: cluster path unavailable on this device
  void* tb = nullptr;        // temporal-blocked solve (ws_sor_tb.cu); null: the colour-list paths
};

// the temporal-blocked solve (ws_sor_tb.cu)
cudaError_t sor_tb_init(void** statePtr, const Dims& d, int device);
void sor_tb_free(void* statePtr);
cudaError_t launch_sor_tb(void* statePtr, const Dims& d, const GridDev& g, const uint8_t* diag8, double omega,
                          int iters, int check, double tol, int* err, int* outIters, double* outRel, int* outPath,
                          cudaStream_t s);
// grids up to this many cells solve on every SM with temporal blocking (at
// 128^3 every region fits in shared memory); larger ones on the colour lists
static const long long kTbMaxCells = 160LL * 160 * 160;

cudaError_t sor_init(void** statePtr, const Dims& d, int device) {
  SorState* S = new SorState();
  *statePtr = S;
  const long long nCells = d.nCells;
  cudaError_t e;
  if (nCells <= kTbMaxCells && (e = sor_tb_init(&S->tb, d, device)) != cudaSuccess) return e;
  int smCount = 0, perSM = 0;
  cudaDeviceGetAttribute(&smCount, cudaDevAttrMultiProcessorCount, device);
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k_sor_persistent, S->block, 0)) != cudaSuccess) return e;
  if (perSM < 1) return cudaErrorLaunchOutOfResources;
  S->grid = std::min(kMaxSorCtas, smCount * (perSM > 1 ? 1 : perSM));
  long long half = nCells / 2 + 2;
  S->cap = half;
  for (int c = 0; c < 2; c++) {
    if ((e = cudaMalloc(&S->L.idx[c], sizeof(int) * half)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&S->L.rhs[c], sizeof(float) * half)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&S->L.pw[c], sizeof(float) * half)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&S->L.dg[c], half)) != cudaSuccess) return e;
  }
  long long nb = (nCells + 255) / 256 + 1;
  for (int c = 0; c < 2; c++)
    if ((e = cudaMalloc(&S->L.code[c], sizeof(uint16_t) * 6 * half)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&S->L.pos, sizeof(int) * nCells)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&S->L.count, sizeof(int) * 2)) != cudaSuccess) return e;
  // the largest cluster this device co-schedules with the solve's shared memory
  size_t smem = cluster_smem_bytes();
  if (cudaFuncSetAttribute(k_sor_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) == cudaSuccess) {
    cudaFuncSetAttribute(k_sor_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    for (int C = kClusterMax; C >= 8 && !S->clusterSize; C /= 2) {
      cudaLaunchConfig_t cfg = {};
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = C; attr[0].val.clusterDim.y = 1; attr[0].val.clusterDim.z = 1;
      cfg.gridDim = dim3(C); cfg.blockDim = dim3(1024); cfg.dynamicSmemBytes = smem;
      cfg.attrs = attr; cfg.numAttrs = 1;
      int nClusters = 0;
      if (cudaOccupancyMaxActiveClusters(&nClusters, k_sor_cluster, &cfg) == cudaSuccess && nClusters >= 1)
        S->clusterSize = C;
    }
  }
  cudaGetLastError();                                   // a refused probe is not an error
  if ((e = cudaMalloc(&S->blockCounts, sizeof(int) * 2 * nb)) != cudaSuccess) return e;
  // zero until the first pressure setup fills them: a solve before it lists no cell
  if ((e = cudaMemset(S->blockCounts, 0, sizeof(int) * 2 * nb)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&S->blockOffs, sizeof(int) * 2 * nb)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&S->bar, sizeof(GridBar))) != cudaSuccess) return e;
  if ((e = cudaMemset(S->bar, 0, sizeof(GridBar))) != cudaSuccess) return e;
  if ((e = cudaMalloc(&S->partials, sizeof(double2) * (S->grid + 1))) != cudaSuccess) return e;
  if ((e = cudaMalloc(&S->outIters, sizeof(int))) != cudaSuccess) return e;
  if ((e = cudaMalloc(&S->outRel, sizeof(double))) != cudaSuccess) return e;
  if ((e = cudaMalloc(&S->outPath, sizeof(int))) != cudaSuccess) return e;
  return cudaSuccess;
}

int* sor_block_counts(void* statePtr) { return statePtr ? ((SorState*)statePtr)->blockCounts : nullptr; }
// kernels one launch_sor_solve issues: scan, scatter, [codes, cluster solve,] grid solve
int sor_solve_launches(void* statePtr) {
  SorState* S = (SorState*)statePtr;
  if (S && S->tb) return 1;
  return S && S->clusterSize ? 5 : 3;
}
bool sor_uses_tb(void* statePtr) { return statePtr && ((SorState*)statePtr)->tb; }
int sor_list_solve_launches(void* statePtr) { return statePtr && ((SorState*)statePtr)->clusterSize ? 5 : 3; }
void sor_free(void* statePtr) {
  SorState* S = (SorState*)statePtr;
  if (!S) return;
  sor_tb_free(S->tb);
  for (int c = 0; c < 2; c++) { cudaFree(S->L.idx[c]); cudaFree(S->L.rhs[c]); cudaFree(S->L.pw[c]); cudaFree(S->L.dg[c]); cudaFree(S->L.code[c]); }
  cudaFree(S->L.pos);
  cudaFree(S->L.count); cudaFree(S->blockCounts); cudaFree(S->blockOffs); cudaFree(S->bar); cudaFree(S->partials);
  cudaFree(S->outIters); cudaFree(S->outRel); cudaFree(S->outPath);
  delete S;
}

// Builds the colour lists from the pressure setup (pw, rhs, diag8) and runs
// the whole solve. Results land in device memory (iterations, residual);
// the caller reads them with its next status synchronisation.
// The colour lists (scan of the setup's block counts, scatter, neighbour
// codes) and the barrier reset. They read the pressure setup's rhs, pw and
// stencil bytes, never q, so they may run beside anything that only writes q
// (the learned warm start).
static cudaError_t build_lists(SorState* S, const Dims& d, const GridDev& g, const uint8_t* diag8, cudaStream_t s);
cudaError_t launch_sor_lists(void* statePtr, const Dims& d, const GridDev& g, const uint8_t* diag8, cudaStream_t s) {
  SorState* S = (SorState*)statePtr;
  if (S->tb) return cudaSuccess;          // the temporal-blocked solve builds its own plan
  return build_lists(S, d, g, diag8, s);
}
static cudaError_t build_lists(SorState* S, const Dims& d, const GridDev& g, const uint8_t* diag8, cudaStream_t s) {
  // the per-block colour counts come from the pressure setup (k_pressure_setup)
  int nb = (int)grid_for(d.nCells, 256);
  k_sor_scan<<<1, 1024, 0, s>>>(S->blockCounts, nb, S->blockOffs, S->L.count);
  k_sor_scatter<<<std::min(nb, 148 * 8), 256, 0, s>>>(d, g.pw, g.rhs, diag8, S->blockOffs, S->L, nb);
  cudaMemsetAsync(S->bar, 0, sizeof(GridBar), s);     // a solve that timed out leaves no stale arrivals
  if (S->clusterSize)
    k_sor_codes<<<dim3((unsigned)std::min<long long>(grid_for(6 * S->cap, 256), 148 * 8), 2), 256, 0, s>>>(d, g.pw,
                                                                                                      S->L, S->clusterSize);
  return cudaGetLastError();
}
// The solve on the lists of launch_sor_lists: cluster-resident when they fit
// one cluster, else the grid-wide persistent kernel (each returns at once when
// the other path applies).
static cudaError_t run_lists(SorState* S, const Dims& d, const GridDev& g, double omega, int iters, int check,
                             double tol, int* err, int** outIters, double** outRel, int** outPath, cudaStream_t s);
cudaError_t launch_sor_run(void* statePtr, const Dims& d, const GridDev& g, const uint8_t* diag8, double omega,
                           int iters, int check, double tol, int* err, int** outIters, double** outRel, int** outPath,
                           cudaStream_t s) {
  SorState* S = (SorState*)statePtr;
  *outPath = S->outPath; *outIters = S->outIters; *outRel = S->outRel;
  if (S->tb)
    return launch_sor_tb(S->tb, d, g, diag8, omega, iters, check, tol, err, S->outIters, S->outRel, S->outPath, s);
  return run_lists(S, d, g, omega, iters, check, tol, err, outIters, outRel, outPath, s);
}
static cudaError_t run_lists(SorState* S, const Dims& d, const GridDev& g, double omega, int iters, int check,
                             double tol, int* err, int** outIters, double** outRel, int** outPath, cudaStream_t s) {
  *outPath = S->outPath;
  int C = S->clusterSize;
  if (C) {
    ClusterArgs ca;
    ca.d = d; ca.q = g.q; ca.L = S->L; ca.om1 = 1 - omega; ca.iters = iters; ca.check = check; ca.tol = tol;
    ca.outIters = S->outIters; ca.outRel = S->outRel; ca.outPath = S->outPath;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C; attr[0].val.clusterDim.y = 1; attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(C); cfg.blockDim = dim3(1024); cfg.dynamicSmemBytes = cluster_smem_bytes();
    cfg.stream = s; cfg.attrs = attr; cfg.numAttrs = 1;
    cudaError_t ec = cudaLaunchKernelEx(&cfg, k_sor_cluster, ca);
    if (ec != cudaSuccess) return ec;
  }
  SorArgs a;
  a.d = d; a.q = g.q; a.L = S->L; a.om1 = 1 - omega; a.iters = iters; a.check = check; a.tol = tol;
  a.bar = S->bar; a.partials = S->partials; a.err = err; a.outIters = S->outIters; a.outRel = S->outRel;
  a.outPath = S->outPath;
  a.clusterCap = C ? C * kSmax : -1;
  a.offs = S->blockOffs; a.nChunks = (int)grid_for(d.nCells, 256);
  void* args[] = { &a };
  cudaError_t e = cudaLaunchCooperativeKernel((void*)k_sor_persistent, dim3(S->grid), dim3(S->block), args, 0, s);
  *outIters = S->outIters; *outRel = S->outRel;
  return e;
}
cudaError_t launch_sor_solve(void* statePtr, const Dims& d, const GridDev& g, const uint8_t* diag8, double omega,
                             int iters, int check, double tol, int* err, int** outIters, double** outRel,
                             int** outPath, cudaStream_t s) {
  cudaError_t e = launch_sor_lists(statePtr, d, g, diag8, s);
  if (e != cudaSuccess) return e;
  return launch_sor_run(statePtr, d, g, diag8, omega, iters, check, tol, err, outIters, outRel, outPath, s);
}
// the same solve on the colour lists (cluster-resident or grid-wide), whatever
// the default path; for comparisons of the two paths
cudaError_t launch_sor_solve_lists(void* statePtr, const Dims& d, const GridDev& g, const uint8_t* diag8, double omega,
                                   int iters, int check, double tol, int* err, int** outIters, double** outRel,
                                   int** outPath, cudaStream_t s) {
  SorState* S = (SorState*)statePtr;
  cudaError_t e = build_lists(S, d, g, diag8, s);
  if (e != cudaSuccess) return e;
  return run_lists(S, d, g, omega, iters, check, tol, err, outIters, outRel, outPath, s);
}
