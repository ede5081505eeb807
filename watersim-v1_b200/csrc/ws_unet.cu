// ws_unet.cu — everything of the warm-start U-Net around the tensor-core
// convolution (ws_unet_conv.cu): tile activity, network input from the
// initial pressure residual, pooling, the output head and loss, the
// backward glue, weight gradients, Adam, and the host driver (class Net).
//
// Network (3 levels, 16/32/64 channels, every conv 3x3x3 + bias + ReLU):
//   L0  e0a = conv(x, 16->16)   s0 = conv(e0a, 16->16)
//   L1  p1 = pool(s0)  e1a = conv(p1, 16->32)  s1 = conv(e1a, 32->32)
//   L2  p2 = pool(s1)  ba = conv(p2, 32->64)   bb = conv(ba, 64->64)
//   L1  d1a = conv(up(bb) | s1, 96->32)        d1b = conv(d1a, 32->32)
//   L0  d0a = conv(up(d1b) | s0, 48->16)       h = conv(d0a, 16->16)
//   out = wh . h + bh  (FP32 head), at fluid cells
// With 4 levels an encoder pair e2a, e2b (32->64, 64->64) sits at L2, the
// bottleneck ba, bb (64->128, 128->128) at L3 and a decoder pair d2a, d2b
// (up(bb) | s2, 192->64; 64->64) at L2.
// pool = 2x2x2 mean, up = nearest x2, | = channel concatenation.
// Input x (16 channels, 4 used): r0 / sigma, fluid, solid, air, where r0 =
// b - A q_prev is the residual of the previous pressure and sigma its RMS
// over fluid cells. The target is (q_converged - q_prev) / (sigma * G), G a
// fixed gain set from the stored pairs, so the network learns the solve's
// correction A^-1 r0 in units independent of the flow's scale.
#include "ws_unet.cuh"
#include <vector>
#include <cmath>
#include <cstring>
#include <algorithm>

namespace unet {

// ------------------------------------------------------------ geometry
__device__ __forceinline__ bool tile_voxel(const Level& L, const int* tiles, int nT, long long i,
                                           int& x, int& y, int& z, long long& v) {
  int ti = (int)(i >> 10);
  if (ti >= nT) return false;
  int t = tiles[ti], r = (int)(i & 1023);
  int tx = t % L.ntx, ty = (t / L.ntx) % L.nty, tz = t / (L.ntx * L.nty);
  x = tx * kTX + (r & 7); y = ty * kTY + ((r >> 3) & 15); z = tz * kTZ + (r >> 7);
  if (x >= L.nx || y >= L.ny || z >= L.nz) return false;
  v = ((long long)z * L.ny + y) * L.nx + x;
  return true;
}
__device__ __forceinline__ bool vox_active(const Level& L, const uint8_t* act, int x, int y, int z) {
  if (x < 0 || y < 0 || z < 0 || x >= L.nx || y >= L.ny || z >= L.nz) return false;
  return act[((z / kTZ) * L.nty + y / kTY) * L.ntx + x / kTX] != 0;
}

// ------------------------------------------------------------ activity
// level-0 tile active <=> it holds a fluid cell; also counts fluid cells
__global__ void k_activity0(Level L, const uint8_t* __restrict__ type, uint8_t* __restrict__ act, int* nFluid) {
  __shared__ int s_any, s_cnt;
  if (threadIdx.x == 0) { s_any = 0; s_cnt = 0; }
  __syncthreads();
  int t = blockIdx.x;
  int tx = t % L.ntx, ty = (t / L.ntx) % L.nty, tz = t / (L.ntx * L.nty);
  int cnt = 0;
  for (int r = threadIdx.x; r < 1024; r += blockDim.x) {
    int x = tx * kTX + (r & 7), y = ty * kTY + ((r >> 3) & 15), z = tz * kTZ + (r >> 7);
    if (x < L.nx && y < L.ny && z < L.nz && type[((long long)z * L.ny + y) * L.nx + x] == WS_FLUID) cnt++;
  }
  cnt = __reduce_add_sync(0xffffffffu, cnt);
  if ((threadIdx.x & 31) == 0 && cnt) { atomicAdd(&s_cnt, cnt); s_any = 1; }
  __syncthreads();
  if (threadIdx.x == 0) { act[t] = (uint8_t)s_any; if (s_cnt) atomicAdd(nFluid, s_cnt); }
}
struct Levels { Level l[kMaxLevels]; uint8_t* act[kMaxLevels]; int* tiles[kMaxLevels]; int* count; int n; };
// one CTA: coarser activity from the finer, then the compacted tile lists
__global__ void k_tile_lists(Levels Ls) {
  __shared__ int wsum[32], carry;
  for (int lv = 0; lv < Ls.n; lv++) {
    const Level& L = Ls.l[lv];
    if (lv > 0) {
      const Level& F = Ls.l[lv - 1];
      for (int t = threadIdx.x; t < L.ntiles; t += blockDim.x) {
        int tx = t % L.ntx, ty = (t / L.ntx) % L.nty, tz = t / (L.ntx * L.nty);
        int a = 0;
        for (int c = 0; c < 8; c++) {
          int fx = 2 * tx + (c & 1), fy = 2 * ty + ((c >> 1) & 1), fz = 2 * tz + (c >> 2);
          if (fx < F.ntx && fy < F.nty && fz < F.ntz) a |= Ls.act[lv - 1][(fz * F.nty + fy) * F.ntx + fx];
        }
        Ls.act[lv][t] = (uint8_t)a;
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < L.ntiles; base += blockDim.x) {
      int t = base + threadIdx.x;
      int a = t < L.ntiles ? Ls.act[lv][t] : 0;
      unsigned m = __ballot_sync(0xffffffffu, a);
      int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
      if (lane == 0) wsum[w] = __popc(m);
      __syncthreads();
      int off = carry;
      for (int k = 0; k < w; k++) off += wsum[k];
      if (a) Ls.tiles[lv][off + __popc(m & ((1u << lane) - 1u))] = t;
      __syncthreads();
      if (threadIdx.x == 0) { int s = 0; for (int k = 0; k < (int)(blockDim.x >> 5); k++) s += wsum[k]; carry += s; }
      __syncthreads();
    }
    if (threadIdx.x == 0) Ls.count[lv] = carry;
    __syncthreads();
  }
}

// ------------------------------------------------------------ input
// r0 = b - A q at fluid cells (FP64; the residual of k_sor_persistent's
// check), block partials of r0^2 -> sigma^2 = sum / nFluid
// over the voxels of the active level-0 tiles only (every fluid cell is in one)
__global__ void k_residual0(Dims d, Level L, const int* tiles, const int* count, const float* __restrict__ q,
                            const float* __restrict__ rhs, const uint8_t* __restrict__ diag8,
                            const uint8_t* __restrict__ type, float* __restrict__ r0, double* __restrict__ partials) {
  __shared__ double ws[32];
  double rr = 0;
  const long long nv = (long long)*count * 1024;
  for (long long iv = blockIdx.x * (long long)blockDim.x + threadIdx.x; iv < nv; iv += (long long)gridDim.x * blockDim.x) {
    int i, j, k; long long c;
    if (!tile_voxel(L, tiles, *count, iv, i, j, k, c)) continue;
    float r = 0.f;
    if (type[c] == WS_FLUID) {
      long long nx = d.nx, nxy = (long long)d.nx * d.ny;
      double s = 0;
      if (i > 0) s += q[c - 1];
      if (i < d.nx - 1) s += q[c + 1];
      if (j > 0) s += q[c - nx];
      if (j < d.ny - 1) s += q[c + nx];
      if (k > 0) s += q[c - nxy];
      if (k < d.nz - 1) s += q[c + nxy];
      double rd = (double)rhs[c] + s - (double)diag8[c] * (double)q[c];
      rr += rd * rd;
      r = (float)rd;
    }
    r0[c] = r;
  }
  for (int o = 16; o; o >>= 1) rr += __shfl_xor_sync(0xffffffffu, rr, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = rr;
  __syncthreads();
  if (threadIdx.x == 0) { double s = 0; for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += ws[w]; partials[blockIdx.x] = s; }
}
// sigma = sqrt(sum / nFluid) (1 if zero); r0 scaled in place by 1/sigma
__global__ void k_sigma(const double* __restrict__ partials, int nb, const int* nFluid, double* sigma) {
  __shared__ double ws[32];
  double s = 0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) s += partials[b];
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0; for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += ws[w];
    int n = *nFluid;
    double sg = n > 0 ? sqrt(t / n) : 0.0;
    *sigma = sg > 0 ? sg : 1.0;
  }
}
__global__ void k_scale(Level L, const int* tiles, const int* count, float* __restrict__ r0, const double* sigma) {
  const long long nv = (long long)*count * 1024;
  for (long long iv = blockIdx.x * (long long)blockDim.x + threadIdx.x; iv < nv; iv += (long long)gridDim.x * blockDim.x) {
    int i, j, k; long long c;
    if (tile_voxel(L, tiles, *count, iv, i, j, k, c)) r0[c] = (float)((double)r0[c] / *sigma);
  }
}
// network input at the voxels of active level-0 tiles
// r0n: the residual already divided by sigma, or (sigma non-null) the raw
// residual, divided here exactly as k_scale would: (float)(r0 / sigma)
__global__ void k_input(Level L, const int* tiles, const int* count, const float* __restrict__ r0n,
                        const uint8_t* __restrict__ type, bf16* __restrict__ x, const double* sigma) {
  const long long n = (long long)*count * 1024;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
  int X, Y, Z; long long v;
  if (!tile_voxel(L, tiles, *count, i, X, Y, Z, v)) continue;
  uint8_t t = type[v];
  bf16 ch[16];
#pragma unroll
  for (int c = 0; c < 16; c++) ch[c] = __float2bfloat16_rn(0.f);
  ch[0] = __float2bfloat16_rn(sigma ? (float)((double)r0n[v] / *sigma) : r0n[v]);
  ch[1] = __float2bfloat16_rn(t == WS_FLUID ? 1.f : 0.f);
  ch[2] = __float2bfloat16_rn(t == WS_SOLID ? 1.f : 0.f);
  ch[3] = __float2bfloat16_rn(t == WS_AIR ? 1.f : 0.f);
  uint4* dst = reinterpret_cast<uint4*>(x + v * 16);
  const uint4* s = reinterpret_cast<const uint4*>(ch);
  dst[0] = s[0]; dst[1] = s[1];
  }
}

// ------------------------------------------------------------ pooling
// coarse voxel = mean of its 8 fine voxels (inactive / outside read as 0)
__global__ void k_pool(Level C, const int* tiles, const int* count, Level F, const uint8_t* __restrict__ factive,
                       const bf16* __restrict__ fine, bf16* __restrict__ coarse, int ch) {
  const long long n = (long long)*count * 1024 * (ch / 8);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
  long long task = i / (ch / 8);
  int c8 = (int)(i % (ch / 8)) * 8;
  int X, Y, Z; long long v;
  if (!tile_voxel(C, tiles, *count, task, X, Y, Z, v)) continue;
  float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int k = 0; k < 8; k++) {
    int fx = 2 * X + (k & 1), fy = 2 * Y + ((k >> 1) & 1), fz = 2 * Z + (k >> 2);
    if (!vox_active(F, factive, fx, fy, fz)) continue;
    uint4 u = __ldg(reinterpret_cast<const uint4*>(fine + (((long long)fz * F.ny + fy) * F.nx + fx) * ch + c8));
    const bf16* b = reinterpret_cast<const bf16*>(&u);
#pragma unroll
    for (int e = 0; e < 8; e++) acc[e] += __bfloat162float(b[e]);
  }
  uint4 o;
  __nv_bfloat162* ob = reinterpret_cast<__nv_bfloat162*>(&o);
#pragma unroll
  for (int e = 0; e < 4; e++) ob[e] = __floats2bfloat162_rn(acc[2 * e] * 0.125f, acc[2 * e + 1] * 0.125f);
  *reinterpret_cast<uint4*>(coarse + v * ch + c8) = o;
  }
}
// backward of pool, added to the skip gradient and masked by the ReLU of s:
// ds(v) = (dskip(v) + dpool(parent) / 8) * (s(v) > 0)
__global__ void k_pool_bwd_add(Level F, const int* tiles, const int* count, Level C,
                               const bf16* __restrict__ dskip, const bf16* __restrict__ dpool,
                               const bf16* __restrict__ s, bf16* __restrict__ ds, int ch) {
  const long long n = (long long)*count * 1024 * (ch / 8);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
  long long task = i / (ch / 8);
  int c8 = (int)(i % (ch / 8)) * 8;
  int X, Y, Z; long long v;
  if (!tile_voxel(F, tiles, *count, task, X, Y, Z, v)) continue;
  long long pv = ((long long)(Z >> 1) * C.ny + (Y >> 1)) * C.nx + (X >> 1);
  uint4 a = __ldg(reinterpret_cast<const uint4*>(dskip + v * ch + c8));
  uint4 b = __ldg(reinterpret_cast<const uint4*>(dpool + pv * ch + c8));
  uint4 m = __ldg(reinterpret_cast<const uint4*>(s + v * ch + c8));
  const bf16 *pa = reinterpret_cast<const bf16*>(&a), *pb = reinterpret_cast<const bf16*>(&b), *pm = reinterpret_cast<const bf16*>(&m);
  float r[8];
#pragma unroll
  for (int e = 0; e < 8; e++)
    r[e] = __bfloat162float(pm[e]) > 0.f ? __bfloat162float(pa[e]) + 0.125f * __bfloat162float(pb[e]) : 0.f;
  uint4 o;
  __nv_bfloat162* ob = reinterpret_cast<__nv_bfloat162*>(&o);
#pragma unroll
  for (int e = 0; e < 4; e++) ob[e] = __floats2bfloat162_rn(r[2 * e], r[2 * e + 1]);
  *reinterpret_cast<uint4*>(ds + v * ch + c8) = o;
  }
}
// backward of the nearest upsampling: coarse gradient = sum over the 8 fine
// children (inactive / outside read as 0), masked by the ReLU of act
__global__ void k_up_bwd(Level C, const int* tiles, const int* count, Level F, const uint8_t* __restrict__ factive,
                         const bf16* __restrict__ dup, const bf16* __restrict__ act, bf16* __restrict__ dc, int ch) {
  const long long n = (long long)*count * 1024 * (ch / 8);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
  long long task = i / (ch / 8);
  int c8 = (int)(i % (ch / 8)) * 8;
  int X, Y, Z; long long v;
  if (!tile_voxel(C, tiles, *count, task, X, Y, Z, v)) continue;
  float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int k = 0; k < 8; k++) {
    int fx = 2 * X + (k & 1), fy = 2 * Y + ((k >> 1) & 1), fz = 2 * Z + (k >> 2);
    if (!vox_active(F, factive, fx, fy, fz)) continue;
    uint4 u = __ldg(reinterpret_cast<const uint4*>(dup + (((long long)fz * F.ny + fy) * F.nx + fx) * ch + c8));
    const bf16* b = reinterpret_cast<const bf16*>(&u);
#pragma unroll
    for (int e = 0; e < 8; e++) acc[e] += __bfloat162float(b[e]);
  }
  uint4 m = __ldg(reinterpret_cast<const uint4*>(act + v * ch + c8));
  const bf16* pm = reinterpret_cast<const bf16*>(&m);
  uint4 o;
  __nv_bfloat162* ob = reinterpret_cast<__nv_bfloat162*>(&o);
#pragma unroll
  for (int e = 0; e < 4; e++)
    ob[e] = __floats2bfloat162_rn(__bfloat162float(pm[2 * e]) > 0.f ? acc[2 * e] : 0.f,
                                  __bfloat162float(pm[2 * e + 1]) > 0.f ? acc[2 * e + 1] : 0.f);
  *reinterpret_cast<uint4*>(dc + v * ch + c8) = o;
  }
}

// ------------------------------------------------------------ output head
// forward: out = wh . h + bh at fluid cells; q += sigma * G * out
__global__ void k_head_apply(Level L, const int* tiles, const int* count, const bf16* __restrict__ h,
                             const float* __restrict__ head, const uint8_t* __restrict__ type,
                             const double* sigma, const double* gain, float* __restrict__ q) {
  const long long n = (long long)*count * 1024;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
  int X, Y, Z; long long v;
  if (!tile_voxel(L, tiles, *count, i, X, Y, Z, v)) continue;
  if (type[v] != WS_FLUID) continue;
  uint4 u[2] = { __ldg(reinterpret_cast<const uint4*>(h + v * 16)), __ldg(reinterpret_cast<const uint4*>(h + v * 16) + 1) };
  const bf16* b = reinterpret_cast<const bf16*>(u);
  float o = head[16];
#pragma unroll
  for (int c = 0; c < 16; c++) o += head[c] * __bfloat162float(b[c]);
  q[v] = (float)((double)q[v] + *sigma * *gain * (double)o);
  }
}
// network output at every active voxel (testing) -> out (fp32, dense)
__global__ void k_head_out(Level L, const int* tiles, const int* count, const bf16* __restrict__ h,
                           const float* __restrict__ head, float* __restrict__ out) {
  const long long n = (long long)*count * 1024;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
  int X, Y, Z; long long v;
  if (!tile_voxel(L, tiles, *count, i, X, Y, Z, v)) continue;
  const bf16* b = h + v * 16;
  float o = head[16];
  for (int c = 0; c < 16; c++) o += head[c] * __bfloat162float(b[c]);
  out[v] = o;
  }
}
// training head: loss = sum_fluid (out - t)^2 / nFluid, its gradients for
// wh, bh (grad[0..16]) and dh = dloss/dout * wh * (h > 0) at every active voxel
__global__ void k_head_train(Level L, const int* tiles, const int* count, const bf16* __restrict__ h,
                             const float* __restrict__ head, const uint8_t* __restrict__ type,
                             const float* __restrict__ target, const int* nFluid,
                             bf16* __restrict__ dh, float* __restrict__ ghead, double* loss) {
  __shared__ float sg[17][8];
  __shared__ double sl[8];
  int X, Y, Z; long long v;
  float g[17];
#pragma unroll
  for (int c = 0; c < 17; c++) g[c] = 0.f;
  double l = 0;
  const long long n = (long long)*count * 1024;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    if (!tile_voxel(L, tiles, *count, i, X, Y, Z, v)) continue;
    const bf16* b = h + v * 16;
    float hv[16];
    float o = head[16];
#pragma unroll
    for (int c = 0; c < 16; c++) { hv[c] = __bfloat162float(b[c]); o += head[c] * hv[c]; }
    float dout = 0.f;
    if (type[v] == WS_FLUID) {
      float diff = o - target[v];
      l += (double)diff * diff;
      dout = 2.f * diff / (float)max(*nFluid, 1);
    }
    bf16 od[16];
#pragma unroll
    for (int c = 0; c < 16; c++) { od[c] = __float2bfloat16_rn(hv[c] > 0.f ? dout * head[c] : 0.f); g[c] += dout * hv[c]; }
    g[16] += dout;
    uint4* dst = reinterpret_cast<uint4*>(dh + v * 16);
    dst[0] = reinterpret_cast<uint4*>(od)[0]; dst[1] = reinterpret_cast<uint4*>(od)[1];
  }
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < 17; c++) {
    float x = g[c];
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) sg[c][w] = x;
  }
  for (int o = 16; o; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if (lane == 0) sl[w] = l;
  __syncthreads();
  if (threadIdx.x < 17) { float s = 0; for (int k = 0; k < (int)(blockDim.x >> 5); k++) s += sg[threadIdx.x][k]; if (s != 0.f) atomicAdd(ghead + threadIdx.x, s); }
  if (threadIdx.x == 32) { double s = 0; for (int k = 0; k < (int)(blockDim.x >> 5); k++) s += sl[k]; if (s != 0) atomicAdd(loss, s / max(*nFluid, 1)); }
}

// ------------------------------------------------------------ weights
// FP32 master W[co][ci][27] -> the packed BF16 operand of the forward conv,
// [ci/16][27][2][co][8], and of the backward-data conv (cin' = co, cout' =
// ci, taps mirrored), [co/16][27][2][ci][8]
// Packed B operands of k_conv3, per 16-channel input slice kk: for each of
// the 9 in-plane taps g = 3 dy + dx, two K halves j (channels 8 j .. 8 j + 7),
// and in each half the rows of the three z taps in the order dz = 2, 1, 0
// (tap t = 9 dz + g), so the rows of consecutive z taps are contiguous along N.
__global__ void k_pack(const float* __restrict__ W, int cin, int cout, bf16* __restrict__ fw, bf16* __restrict__ bw) {
  int n = 27 * cin * cout;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  {  // forward: i = (((((kk * 9 + g) * 2 + j) * 3 + (2 - dz)) * cout + co) * 8 + e)
    int e = i & 7, r = i >> 3;
    int co = r % cout; r /= cout;
    int dz = 2 - r % 3; r /= 3;
    int j = r & 1; r >>= 1;
    int g = r % 9, kk = r / 9;
    fw[i] = __float2bfloat16_rn(W[((size_t)co * cin + kk * 16 + j * 8 + e) * 27 + 9 * dz + g]);
  }
  {  // backward data: the same layout over ci, co = 16 kk + 8 j + e, taps mirrored
    int e = i & 7, r = i >> 3;
    int ci = r % cin; r /= cin;
    int dz = 2 - r % 3; r /= 3;
    int j = r & 1; r >>= 1;
    int g = r % 9, kk = r / 9;
    bw[i] = __float2bfloat16_rn(W[((size_t)(kk * 16 + j * 8 + e) * cin + ci) * 27 + (26 - (9 * dz + g))]);
  }
}
// Adam (Kingma & Ba 2015) on the flat FP32 parameter vector; grad is the sum
// over the batch, scaled by 1/batch here
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       long long n, float lr, float b1, float b2, float eps, float c1, float c2, float inv_batch) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  float gi = g[i] * inv_batch;
  float mi = b1 * m[i] + (1.f - b1) * gi;
  float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi; v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// ------------------------------------------------------------ training pairs
// after the solve: target = (q - q_prev) / sigma at fluid cells, 0 elsewhere;
// t2 += sum target^2 (for the gain)
__global__ void k_pair_target(long long n, const float* __restrict__ q, const float* __restrict__ qprev,
                              const uint8_t* __restrict__ type, const double* sigma, float* __restrict__ target,
                              double* t2) {
  __shared__ double ws[32];
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double s = 0;
  if (c < n) {
    float t = 0.f;
    if (type[c] == WS_FLUID) { double d = ((double)q[c] - (double)qprev[c]) / *sigma; t = (float)d; s = d * d; }
    target[c] = t;
  }
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) { double t = 0; for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += ws[w]; if (t != 0) atomicAdd(t2, t); }
}
// target scaled by 1/G for the loss
__global__ void k_scale_copy(const float* __restrict__ a, float* __restrict__ b, long long n, float s) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c < n) b[c] = a[c] * s;
}
// A pair slot holds, for each of its tiles k (tile id stiles[k]), the 1024
// voxels of that level-0 tile in tile order (r = x + 8 (y + 16 z)).
// pack: dense level-0 arrays -> slot, over the tile list of the current
// activity (tiles, *count). With r0 / type null only the target is packed.
__global__ void k_pair_pack(Level L, const int* __restrict__ tiles, const int* count, int tileCap,
                            const float* __restrict__ r0, const uint8_t* __restrict__ type,
                            const float* __restrict__ target, float* __restrict__ sr0, uint8_t* __restrict__ stype,
                            float* __restrict__ starget, int* __restrict__ stiles) {
  const int nT = *count;
  if (nT > tileCap) return;                        // the slot is marked unusable by the host
  const long long n = (long long)nT * 1024;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    if ((i & 1023) == 0 && stiles) stiles[i >> 10] = tiles[i >> 10];
    int X, Y, Z; long long v;
    const bool in = tile_voxel(L, tiles, nT, i, X, Y, Z, v);
    if (r0) sr0[i] = in ? r0[v] : 0.f;
    if (type) stype[i] = in ? type[v] : (uint8_t)WS_AIR;
    if (target) starget[i] = in ? target[v] : 0.f;
  }
}
// unpack slot -> dense level-0 arrays at its tiles, and the level-0 activity
__global__ void k_pair_unpack(Level L, const int* __restrict__ stiles, const int* __restrict__ meta,
                              const float* __restrict__ sr0, const uint8_t* __restrict__ stype,
                              const float* __restrict__ starget, float* __restrict__ r0, uint8_t* __restrict__ type,
                              float* __restrict__ target, uint8_t* __restrict__ act0, int* fluidCount) {
  const int nT = meta[0];
  const long long n = (long long)nT * 1024;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    if ((i & 1023) == 0) act0[stiles[i >> 10]] = 1;
    if (i == 0) *fluidCount = meta[1];
    int X, Y, Z; long long v;
    if (!tile_voxel(L, stiles, nT, i, X, Y, Z, v)) continue;
    if (r0) r0[v] = sr0[i];
    type[v] = stype[i];
    if (target) target[v] = starget[i];
  }
}

// ------------------------------------------------------------ host driver
static inline unsigned grid1(long long n, int b) { return (unsigned)((n + b - 1) / b); }
// grid of a grid-stride kernel over at most n items: a few waves of the device
static inline unsigned gridv(long long n, int b) { return (unsigned)std::min<long long>(grid1(n, b), 148LL * 8); }

// He-normal initial weights from a seeded LCG and Box-Muller (host)
struct HostRng {
  uint64_t s;
  explicit HostRng(uint64_t seed) : s(seed * 6364136223846793005ull + 1442695040888963407ull) {}
  uint32_t next() { s = s * 6364136223846793005ull + 1442695040888963407ull; return (uint32_t)(s >> 33); }
  double normal() {
    double u1 = (next() + 0.5) / 4294967296.0, u2 = (next() + 0.5) / 4294967296.0;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
};

int unet_layers(int levels, LayerSpec* out) {
  static const char* encA[] = { "e0a", "e1a", "e2a" };
  static const char* encB[] = { "e0b", "e1b", "e2b" };
  static const char* decA[] = { "d0a", "d1a", "d2a" };
  static const char* decB[] = { "d0b", "d1b", "d2b" };
  int n = 0;
  for (int l = 0; l + 1 < levels; l++) {
    const int c = 16 << l, cin = l == 0 ? 16 : 16 << (l - 1);
    out[n++] = { encA[l], l, 0, cin, c };
    out[n++] = { encB[l], l, 0, c, c };
  }
  const int cb = 16 << (levels - 1);
  out[n++] = { "ba", levels - 1, 0, cb / 2, cb };
  out[n++] = { "bb", levels - 1, 0, cb, cb };
  for (int l = levels - 2; l >= 0; l--) {
    const int c = 16 << l;
    out[n++] = { decA[l], l, 2 * c, c, c };
    out[n++] = { decB[l], l, 0, c, c };
  }
  return n;
}

long long Net::layer_weights(int l) const { return 27LL * (layers[l].c0 + layers[l].c1) * layers[l].cout; }

cudaError_t Net::create(const Dims& d, int nlev) {
  cudaError_t e;
  if (nlev < 3 || nlev > kMaxLevels) return cudaErrorInvalidValue;
  dims = d;
  levels = nlev;
  nLayers = unet_layers(levels, layers);
  int nx = d.nx, ny = d.ny, nz = d.nz;
  for (int l = 0; l < levels; l++) {
    Level& L = lv[l];
    L.nx = nx; L.ny = ny; L.nz = nz;
    L.ntx = (nx + kTX - 1) / kTX; L.nty = (ny + kTY - 1) / kTY; L.ntz = (nz + kTZ - 1) / kTZ;
    L.ntiles = L.ntx * L.nty * L.ntz;
    L.nvox = (long long)nx * ny * nz;
    if ((e = cudaMalloc(&act[l], L.ntiles)) != cudaSuccess) return e;
    if ((e = cudaMemset(act[l], 0, L.ntiles)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&tiles[l], sizeof(int) * L.ntiles)) != cudaSuccess) return e;
    nx = (nx + 1) / 2; ny = (ny + 1) / 2; nz = (nz + 1) / 2;
  }
  if ((e = cudaMalloc(&counts, sizeof(int) * (kMaxLevels + 1))) != cudaSuccess) return e;   // tile counts + fluid count
  if ((e = cudaMemset(counts, 0, sizeof(int) * (kMaxLevels + 1))) != cudaSuccess) return e;
  // parameters
  nparams = 0;
  for (int l = 0; l < nLayers; l++) { woff[l] = nparams; nparams += layer_weights(l); boff[l] = nparams; nparams += layers[l].cout; }
  headOff = nparams; nparams += 17;
  if ((e = cudaMalloc(&params, sizeof(float) * nparams)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&grads, sizeof(float) * nparams)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&adm, sizeof(float) * nparams)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&adv, sizeof(float) * nparams)) != cudaSuccess) return e;
  for (int l = 0; l < nLayers; l++) {
    if ((e = cudaMalloc(&fw[l], sizeof(bf16) * layer_weights(l))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&bw[l], sizeof(bf16) * layer_weights(l))) != cudaSuccess) return e;
  }
  // activations and gradients (NDHWC bf16, dense per level)
  auto A = [&](bf16** p, int l, int c) -> cudaError_t {
    cudaError_t r = cudaMalloc(p, sizeof(bf16) * lv[l].nvox * c);
    if (r == cudaSuccess) r = cudaMemset(*p, 0, sizeof(bf16) * lv[l].nvox * c);
    return r;
  };
  const int L1 = levels - 1;
  if ((e = A(&x, 0, 16)) != cudaSuccess) return e;
  for (int l = 0; l < L1; l++) {
    bf16** same[] = { &ea[l], &sk[l], &da[l], &db[l], &gdb[l], &gda[l], &gsa[l], &gs[l], &gea[l] };
    for (bf16** p : same) if ((e = A(p, l, ch(l))) != cudaSuccess) return e;
    if ((e = A(&gup[l], l, ch(l + 1))) != cudaSuccess) return e;
    if ((e = A(&pl[l + 1], l + 1, ch(l))) != cudaSuccess) return e;
    if ((e = A(&gp[l + 1], l + 1, ch(l))) != cudaSuccess) return e;
  }
  bf16** bot[] = { &bA, &bB, &gbA, &gbB };
  for (bf16** p : bot) if ((e = A(p, L1, ch(L1))) != cudaSuccess) return e;
  long long N = d.nCells;
  nPartials = (int)grid1(N, 256);
  if ((e = cudaMalloc(&partials, sizeof(double) * nPartials)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&scal, sizeof(double) * 8)) != cudaSuccess) return e;   // sigma, gain, loss, t2
  if ((e = cudaMemset(scal, 0, sizeof(double) * 8)) != cudaSuccess) return e;
  float** fbufs[] = { &r0n, &qprev, &tscaled, &outbuf, &tbuf };
  for (float** p : fbufs) {
    if ((e = cudaMalloc(p, sizeof(float) * N)) != cudaSuccess) return e;
    if ((e = cudaMemset(*p, 0, sizeof(float) * N)) != cudaSuccess) return e;
  }
  if ((e = cudaMalloc(&typebuf, (size_t)N)) != cudaSuccess) return e;
  if ((e = cudaMemset(typebuf, 0, (size_t)N)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&err, sizeof(int))) != cudaSuccess) return e;
  if ((e = cudaMemset(err, 0, sizeof(int))) != cudaSuccess) return e;
  return conv3_init();
}

void Net::destroy() {
  void* bufs[] = { counts, params, grads, adm, adv, x, bA, bB, gbA, gbB, partials, scal, r0n, qprev, tscaled, outbuf,
                   tbuf, typebuf, err, pr0n, ptype, ptarget, ptiles, pmeta, pscal };
  for (void* b : bufs) if (b) cudaFree(b);
  for (int l = 0; l < kMaxLevels; l++) {
    void* per[] = { act[l], tiles[l], ea[l], sk[l], pl[l], da[l], db[l], gdb[l], gda[l], gup[l], gsa[l], gp[l], gs[l],
                    gea[l] };
    for (void* b : per) if (b) cudaFree(b);
  }
  for (int l = 0; l < kMaxLayers; l++) { if (fw[l]) cudaFree(fw[l]); if (bw[l]) cudaFree(bw[l]); }
}

cudaError_t Net::init_weights(uint32_t seed, cudaStream_t s) {
  std::vector<float> P((size_t)nparams, 0.f);
  HostRng rng(seed);
  for (int l = 0; l < nLayers; l++) {
    int cin = layers[l].c0 + layers[l].c1;
    double sd = std::sqrt(2.0 / (27.0 * cin));
    for (long long i = 0; i < layer_weights(l); i++) P[(size_t)(woff[l] + i)] = (float)(sd * rng.normal());
  }
  for (int c = 0; c < 16; c++) P[(size_t)(headOff + c)] = (float)(0.25 * rng.normal());
  cudaError_t e;
  if ((e = cudaMemcpyAsync(params, P.data(), sizeof(float) * nparams, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(adm, 0, sizeof(float) * nparams, s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(adv, 0, sizeof(float) * nparams, s)) != cudaSuccess) return e;
  adamStep = 0; trainSteps = 0;
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
  return pack(s);
}
cudaError_t Net::set_weights(const float* host, cudaStream_t s) {
  cudaError_t e = cudaMemcpyAsync(params, host, sizeof(float) * nparams, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
  return pack(s);
}
cudaError_t Net::pack(cudaStream_t s) {
  for (int l = 0; l < nLayers; l++) {
    int n = (int)layer_weights(l);
    k_pack<<<grid1(n, 256), 256, 0, s>>>(params + woff[l], layers[l].c0 + layers[l].c1, layers[l].cout, fw[l], bw[l]);
  }
  return cudaGetLastError();
}

// the coarser levels' activity and every level's tile list from act[0]
cudaError_t Net::lists(cudaStream_t s) {
  Levels Ls;
  for (int l = 0; l < levels; l++) { Ls.l[l] = lv[l]; Ls.act[l] = act[l]; Ls.tiles[l] = tiles[l]; }
  Ls.count = counts; Ls.n = levels;
  k_tile_lists<<<1, 1024, 0, s>>>(Ls);
  return cudaGetLastError();
}
// tile activity of all levels from cell types; counts[kMaxLevels] = fluid cells
cudaError_t Net::activity(const uint8_t* type, cudaStream_t s) {
  cudaMemsetAsync(counts + kMaxLevels, 0, sizeof(int), s);
  k_activity0<<<lv[0].ntiles, 256, 0, s>>>(lv[0], type, act[0], counts + kMaxLevels);
  return lists(s);
}

cudaError_t Net::conv(int l, const bf16* src0, const bf16* src1, bf16* out, cudaStream_t s) {
  const LayerSpec& S = layers[l];
  const Level& L = lv[S.level];
  ConvArgs a{};
  a.nx = L.nx; a.ny = L.ny; a.nz = L.nz; a.ntx = L.ntx; a.nty = L.nty; a.ntz = L.ntz;
  a.tiles = tiles[S.level]; a.nTiles = counts + S.level; a.active = act[S.level];
  a.src0 = src0; a.c0 = S.c0; a.up0 = S.c0 > 0; a.src1 = src1; a.c1 = S.c1;
  a.w = fw[l]; a.bias = params + boff[l]; a.mode = 0; a.mask = nullptr;
  a.out0 = out; a.split = S.cout; a.out1 = nullptr; a.err = err;
  return launch_conv3(a, S.cout, L.ntiles, s);
}
// backward data of layer l: dX = conv^T(dZ), optionally masked by (mask > 0)
// or split into the upsampled part (out0) and the skip part (out1)
cudaError_t Net::conv_bwd(int l, const bf16* dz, const bf16* mask, bf16* out0, bf16* out1, cudaStream_t s) {
  const LayerSpec& S = layers[l];
  const Level& L = lv[S.level];
  ConvArgs a{};
  a.nx = L.nx; a.ny = L.ny; a.nz = L.nz; a.ntx = L.ntx; a.nty = L.nty; a.ntz = L.ntz;
  a.tiles = tiles[S.level]; a.nTiles = counts + S.level; a.active = act[S.level];
  a.src0 = nullptr; a.c0 = 0; a.up0 = 0; a.src1 = dz; a.c1 = S.cout;
  a.w = bw[l]; a.bias = nullptr; a.mode = 1; a.mask = mask;
  const int cin = S.c0 + S.c1;
  a.out0 = out0; a.split = S.c0 > 0 ? S.c0 : cin; a.out1 = out1; a.err = err;
  return launch_conv3(a, cin, L.ntiles, s);
}
cudaError_t Net::dw(int l, const bf16* src0, const bf16* src1, const bf16* dz, cudaStream_t s) {
  const LayerSpec& S = layers[l];
  const Level& L = lv[S.level];
  ConvArgs a{};
  a.nx = L.nx; a.ny = L.ny; a.nz = L.nz; a.ntx = L.ntx; a.nty = L.nty; a.ntz = L.ntz;
  a.tiles = tiles[S.level]; a.nTiles = counts + S.level; a.active = act[S.level];
  a.src0 = src0; a.c0 = S.c0; a.up0 = S.c0 > 0; a.src1 = src1; a.c1 = S.c1; a.err = err;
  const int cin = S.c0 + S.c1;
  return launch_dw_tc(a, dz, S.cout, grads + woff[l], grads + boff[l], L.ntiles * (cin / 16), s);
}

cudaError_t Net::pool(int fineLevel, const bf16* fine, bf16* coarse, int c, cudaStream_t s) {
  const Level& C = lv[fineLevel + 1];
  long long n = (long long)C.ntiles * 1024 * (c / 8);
  k_pool<<<gridv(n, 256), 256, 0, s>>>(C, tiles[fineLevel + 1], counts + fineLevel + 1, lv[fineLevel], act[fineLevel],
                                       fine, coarse, c);
  return cudaGetLastError();
}

// forward pass on the input already in x (activity and tile lists built)
cudaError_t Net::forward(cudaStream_t s) {
  cudaError_t e;
  const bf16* cur = x;
  for (int l = 0; l + 1 < levels; l++) {
    if ((e = conv(enc_a(l), nullptr, cur, ea[l], s)) != cudaSuccess) return e;
    if ((e = conv(enc_b(l), nullptr, ea[l], sk[l], s)) != cudaSuccess) return e;
    if ((e = pool(l, sk[l], pl[l + 1], ch(l), s)) != cudaSuccess) return e;
    cur = pl[l + 1];
  }
  if ((e = conv(bot_a(), nullptr, cur, bA, s)) != cudaSuccess) return e;
  if ((e = conv(bot_b(), nullptr, bA, bB, s)) != cudaSuccess) return e;
  const bf16* up = bB;
  for (int l = levels - 2; l >= 0; l--) {
    if ((e = conv(dec_a(l), up, sk[l], da[l], s)) != cudaSuccess) return e;
    if ((e = conv(dec_b(l), nullptr, da[l], db[l], s)) != cudaSuccess) return e;
    up = db[l];
  }
  return cudaSuccess;
}

// backward pass from the head gradient in gdb[0]; accumulates into grads
cudaError_t Net::backward(cudaStream_t s) {
  cudaError_t e;
  auto upb = [&](int coarseLevel, const bf16* dup, const bf16* a, bf16* out, int c) {
    const Level& C = lv[coarseLevel];
    long long n = (long long)C.ntiles * 1024 * (c / 8);
    k_up_bwd<<<gridv(n, 256), 256, 0, s>>>(C, tiles[coarseLevel], counts + coarseLevel, lv[coarseLevel - 1],
                                           act[coarseLevel - 1], dup, a, out, c);
    return cudaGetLastError();
  };
  auto pba = [&](int fineLevel, const bf16* dskip, const bf16* dpool, const bf16* sAct, bf16* out, int c) {
    const Level& F = lv[fineLevel];
    long long n = (long long)F.ntiles * 1024 * (c / 8);
    k_pool_bwd_add<<<gridv(n, 256), 256, 0, s>>>(F, tiles[fineLevel], counts + fineLevel, lv[fineLevel + 1],
                                                 dskip, dpool, sAct, out, c);
    return cudaGetLastError();
  };
  const int L1 = levels - 1;
  // decoder, from level 0 up: d<l>b, then d<l>a and the gradient of what it upsampled
  for (int l = 0; l < L1; l++) {
    if ((e = dw(dec_b(l), nullptr, da[l], gdb[l], s)) != cudaSuccess) return e;
    if ((e = conv_bwd(dec_b(l), gdb[l], da[l], gda[l], nullptr, s)) != cudaSuccess) return e;
    const bf16* upSrc = l + 1 < L1 ? db[l + 1] : bB;
    if ((e = dw(dec_a(l), upSrc, sk[l], gda[l], s)) != cudaSuccess) return e;
    if ((e = conv_bwd(dec_a(l), gda[l], nullptr, gup[l], gsa[l], s)) != cudaSuccess) return e;
    if ((e = upb(l + 1, gup[l], upSrc, l + 1 < L1 ? gdb[l + 1] : gbB, ch(l + 1))) != cudaSuccess) return e;
  }
  // bottleneck
  if ((e = dw(bot_b(), nullptr, bA, gbB, s)) != cudaSuccess) return e;
  if ((e = conv_bwd(bot_b(), gbB, bA, gbA, nullptr, s)) != cudaSuccess) return e;
  if ((e = dw(bot_a(), nullptr, pl[L1], gbA, s)) != cudaSuccess) return e;
  if ((e = conv_bwd(bot_a(), gbA, nullptr, gp[L1], nullptr, s)) != cudaSuccess) return e;
  // encoder, from the deepest level down
  for (int l = L1 - 1; l >= 0; l--) {
    if ((e = pba(l, gsa[l], gp[l + 1], sk[l], gs[l], ch(l))) != cudaSuccess) return e;
    if ((e = dw(enc_b(l), nullptr, ea[l], gs[l], s)) != cudaSuccess) return e;
    if ((e = conv_bwd(enc_b(l), gs[l], ea[l], gea[l], nullptr, s)) != cudaSuccess) return e;
    if ((e = dw(enc_a(l), nullptr, l == 0 ? x : pl[l], gea[l], s)) != cudaSuccess) return e;
    if (l > 0 && (e = conv_bwd(enc_a(l), gea[l], nullptr, gp[l], nullptr, s)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// r0 / sigma of the current pressure setup into dst, sigma into sig
cudaError_t Net::residual(const float* q, const float* rhs, const uint8_t* diag8, const uint8_t* type,
                          float* dst, double* sig, cudaStream_t s, bool scale) {
  const long long n = (long long)lv[0].ntiles * 1024;
  const unsigned nb = std::min<unsigned>(gridv(n, 256), (unsigned)nPartials);
  k_residual0<<<nb, 256, 0, s>>>(dims, lv[0], tiles[0], counts, q, rhs, diag8, type, dst, partials);
  k_sigma<<<1, 1024, 0, s>>>(partials, (int)nb, counts + kMaxLevels, sig);
  if (scale) k_scale<<<gridv(n, 256), 256, 0, s>>>(lv[0], tiles[0], counts, dst, sig);
  return cudaGetLastError();
}

// learned warm start: q += sigma G net(r0 / sigma, types) at fluid cells
cudaError_t Net::predict(float* q, const float* rhs, const uint8_t* diag8, const uint8_t* type, cudaStream_t s) {
  cudaError_t e;
  if ((e = activity(type, s)) != cudaSuccess) return e;          // also the fluid count sigma divides by
  // raw residual; k_input divides by sigma at the active voxels only
  if ((e = residual(q, rhs, diag8, type, r0n, scal + 0, s, false)) != cudaSuccess) return e;
  long long n = (long long)lv[0].ntiles * 1024;
  k_input<<<gridv(n, 256), 256, 0, s>>>(lv[0], tiles[0], counts, r0n, type, x, scal + 0);
  if ((e = forward(s)) != cudaSuccess) return e;
  k_head_apply<<<gridv(n, 256), 256, 0, s>>>(lv[0], tiles[0], counts, db[0], params + headOff, type, scal + 0, scal + 1, q);
  return cudaGetLastError();
}

// ---- training pairs
// A slot holds tileCap level-0 tiles: every tile when the grid has at most
// 2048 of them, else 1.5 x the active tiles of the current cell types (at
// least 256). A pair with more active tiles is not stored (pairsDropped).
cudaError_t Net::reserve_pairs(int capacity, const uint8_t* type, cudaStream_t s) {
  if (capacity <= pairCap) return cudaSuccess;
  cudaError_t e;
  int cap = lv[0].ntiles;
  if (cap > 2048) {
    if ((e = activity(type, s)) != cudaSuccess) return e;
    int c0 = 0;
    if ((e = cudaMemcpyAsync(&c0, counts, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
    cap = std::min(lv[0].ntiles, std::max(256, c0 + c0 / 2));
  }
  if (tileCap > 0) cap = tileCap;                 // slots keep their size once made
  const size_t V = (size_t)cap * 1024;
  float *a = nullptr, *c = nullptr; uint8_t* b = nullptr; int *t = nullptr, *m = nullptr; double* sc = nullptr;
  if ((e = cudaMalloc(&a, sizeof(float) * V * capacity)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&b, V * capacity)) != cudaSuccess) { cudaFree(a); return e; }
  if ((e = cudaMalloc(&c, sizeof(float) * V * capacity)) != cudaSuccess) { cudaFree(a); cudaFree(b); return e; }
  if ((e = cudaMalloc(&t, sizeof(int) * (size_t)cap * capacity)) != cudaSuccess) { cudaFree(a); cudaFree(b); cudaFree(c); return e; }
  if ((e = cudaMalloc(&m, sizeof(int) * 2 * capacity)) != cudaSuccess) { cudaFree(a); cudaFree(b); cudaFree(c); cudaFree(t); return e; }
  if ((e = cudaMalloc(&sc, sizeof(double) * 2 * capacity)) != cudaSuccess) {
    cudaFree(a); cudaFree(b); cudaFree(c); cudaFree(t); cudaFree(m); return e;
  }
  cudaMemset(sc, 0, sizeof(double) * 2 * capacity);
  cudaMemset(m, 0, sizeof(int) * 2 * capacity);
  if (pairCap > 0 && pairsStored > 0) {           // keep the stored pairs
    const int keep = std::min(pairsStored, pairCap);
    cudaMemcpy(a, pr0n, sizeof(float) * V * keep, cudaMemcpyDeviceToDevice);
    cudaMemcpy(b, ptype, V * keep, cudaMemcpyDeviceToDevice);
    cudaMemcpy(c, ptarget, sizeof(float) * V * keep, cudaMemcpyDeviceToDevice);
    cudaMemcpy(t, ptiles, sizeof(int) * (size_t)cap * keep, cudaMemcpyDeviceToDevice);
    cudaMemcpy(m, pmeta, sizeof(int) * 2 * keep, cudaMemcpyDeviceToDevice);
    cudaMemcpy(sc, pscal, sizeof(double) * 2 * keep, cudaMemcpyDeviceToDevice);
  }
  void* old[] = { pr0n, ptype, ptarget, ptiles, pmeta, pscal };
  for (void* o : old) if (o) cudaFree(o);
  pr0n = a; ptype = b; ptarget = c; ptiles = t; pmeta = m; pscal = sc; pairCap = capacity; tileCap = cap;
  return cudaSuccess;
}
// before the solve: slot <- (r0 / sigma, types) over the active tiles, q_prev saved
cudaError_t Net::collect_pre(const float* q, const float* rhs, const uint8_t* diag8, const uint8_t* type, cudaStream_t s) {
  if (pairCap <= 0) return cudaSuccess;
  const int slot = pairsStored % pairCap;
  const size_t V = (size_t)tileCap * 1024;
  cudaError_t e;
  if ((e = activity(type, s)) != cudaSuccess) return e;
  if ((e = residual(q, rhs, diag8, type, r0n, pscal + 2 * slot, s)) != cudaSuccess) return e;
  int c[2];                                        // active level-0 tiles, fluid cells
  if ((e = cudaMemcpyAsync(&c[0], counts, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(&c[1], counts + kMaxLevels, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
  if (c[0] > tileCap) { pendingSlot = -1; pairsDropped++; return cudaSuccess; }
  k_pair_pack<<<gridv((long long)c[0] * 1024, 256), 256, 0, s>>>(lv[0], tiles[0], counts, tileCap, r0n, type, nullptr,
                                                                pr0n + V * slot, ptype + V * slot, nullptr,
                                                                ptiles + (size_t)tileCap * slot);
  if ((e = cudaMemcpyAsync(pmeta + 2 * slot, c, sizeof(c), cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;   // c lives on this frame
  pendingSlot = slot;
  cudaMemcpyAsync(typebuf, type, (size_t)dims.nCells, cudaMemcpyDeviceToDevice, s);
  cudaMemcpyAsync(qprev, q, sizeof(float) * dims.nCells, cudaMemcpyDeviceToDevice, s);
  return cudaGetLastError();
}
// after the solve: target = (q - q_prev) / sigma over the slot's tiles
cudaError_t Net::collect_post(const float* q, cudaStream_t s) {
  if (pairCap <= 0 || pendingSlot < 0) return cudaSuccess;
  const int slot = pendingSlot;
  const size_t V = (size_t)tileCap * 1024;
  long long N = dims.nCells;
  cudaMemsetAsync(pscal + 2 * slot + 1, 0, sizeof(double), s);
  k_pair_target<<<grid1(N, 256), 256, 0, s>>>(N, q, qprev, typebuf, pscal + 2 * slot, tbuf, pscal + 2 * slot + 1);
  // the activity (and so tiles[0]) still describes the pre-solve types
  k_pair_pack<<<gridv((long long)tileCap * 1024, 256), 256, 0, s>>>(lv[0], tiles[0], counts, tileCap, nullptr, nullptr,
                                                                   tbuf, nullptr, nullptr, ptarget + V * slot, nullptr);
  pairsStored++;
  pendingSlot = -1;
  return cudaGetLastError();
}
// slot p -> the dense level-0 inputs (r0n, typebuf, tbuf) at its tiles, the activity and tile lists
cudaError_t Net::unpack(int p, cudaStream_t s) {
  const size_t V = (size_t)tileCap * 1024;
  cudaError_t e;
  if ((e = cudaMemsetAsync(act[0], 0, lv[0].ntiles, s)) != cudaSuccess) return e;
  k_pair_unpack<<<gridv((long long)tileCap * 1024, 256), 256, 0, s>>>(lv[0], ptiles + (size_t)tileCap * p, pmeta + 2 * p,
                                                                     pr0n + V * p, ptype + V * p, ptarget + V * p,
                                                                     r0n, typebuf, tbuf, act[0], counts + kMaxLevels);
  if ((e = lists(s)) != cudaSuccess) return e;
  long long n = (long long)lv[0].ntiles * 1024;
  k_input<<<gridv(n, 256), 256, 0, s>>>(lv[0], tiles[0], counts, r0n, typebuf, x, nullptr);
  return cudaGetLastError();
}

// gain G = RMS of the stored targets over fluid cells (set once, before the first training step)
cudaError_t Net::set_gain_from_pairs(cudaStream_t s) {
  const int n = stored();
  if (n <= 0) return cudaErrorInvalidValue;
  std::vector<double> sc((size_t)2 * n);
  std::vector<int> meta((size_t)2 * n);
  cudaError_t e = cudaMemcpyAsync(sc.data(), pscal, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(meta.data(), pmeta, sizeof(int) * 2 * n, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
  double t2 = 0, cnt = 0;
  for (int p = 0; p < n; p++) { t2 += sc[(size_t)2 * p + 1]; cnt += meta[(size_t)2 * p + 1]; }
  return set_gain(cnt > 0 && t2 > 0 ? std::sqrt(t2 / cnt) : 1.0, s);
}

cudaError_t Net::set_gain(double g, cudaStream_t s) {
  gain = g;
  cudaError_t e = cudaMemcpyAsync(scal + 1, &gain, sizeof(double), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(s);
}
// one sample: forward + loss + backward into grads (grads not cleared)
cudaError_t Net::sample_grad(int p, cudaStream_t s) {
  long long N = dims.nCells;
  cudaError_t e;
  if ((e = unpack(p, s)) != cudaSuccess) return e;
  if ((e = forward(s)) != cudaSuccess) return e;
  k_scale_copy<<<grid1(N, 256), 256, 0, s>>>(tbuf, tscaled, N, (float)(1.0 / gain));
  long long n = (long long)lv[0].ntiles * 1024;
  k_head_train<<<gridv(n, 256), 256, 0, s>>>(lv[0], tiles[0], counts, db[0], params + headOff, typebuf, tscaled,
                                             counts + kMaxLevels, gdb[0], grads + headOff, scal + 2);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  return backward(s);
}
// zero the gradients and the loss, then add the gradients of `samples`
// pairs drawn with a seeded generator (no parameter update)
cudaError_t Net::accumulate(int samples, uint32_t seed, cudaStream_t s) {
  const int n = stored();
  if (n <= 0 || samples < 0) return cudaErrorInvalidValue;
  cudaError_t e;
  if (!(gain > 0)) { if ((e = set_gain_from_pairs(s)) != cudaSuccess) return e; }
  HostRng rng(seed ? seed : 1u);
  cudaMemsetAsync(grads, 0, sizeof(float) * nparams, s);
  cudaMemsetAsync(scal + 2, 0, sizeof(double), s);
  for (int b = 0; b < samples; b++)
    if ((e = sample_grad((int)(rng.next() % (uint32_t)n), s)) != cudaSuccess) return e;
  return cudaSuccess;
}
// one Adam step with the accumulated gradients divided by `total` samples
cudaError_t Net::apply(double lr, int total, cudaStream_t s) {
  if (total < 1) return cudaErrorInvalidValue;
  adamStep++;
  const float b1 = 0.9f, b2 = 0.999f;
  float c1 = 1.f - std::pow(b1, (float)adamStep), c2 = 1.f - std::pow(b2, (float)adamStep);
  k_adam<<<grid1(nparams, 256), 256, 0, s>>>(params, grads, adm, adv, nparams, (float)lr, b1, b2, 1e-8f, c1, c2,
                                           1.f / total);
  cudaError_t e = pack(s);
  if (e == cudaSuccess) trainSteps++;
  return e;
}
cudaError_t Net::loss_sum(double* out, cudaStream_t s) {
  cudaError_t e = cudaMemcpyAsync(out, scal + 2, sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(s);
}
cudaError_t Net::train(int steps, int batch, double lr, uint32_t seed, double* meanLoss, cudaStream_t s) {
  const int n = stored();
  if (n <= 0 || steps < 0 || batch < 1) return cudaErrorInvalidValue;
  cudaError_t e;
  if (!(gain > 0)) { if ((e = set_gain_from_pairs(s)) != cudaSuccess) return e; }
  HostRng rng(seed ? seed : 1u);
  double total = 0;
  for (int it = 0; it < steps; it++) {
    if ((e = accumulate(batch, rng.next() | 1u, s)) != cudaSuccess) return e;
    if ((e = apply(lr, batch, s)) != cudaSuccess) return e;
    double L = 0;
    if ((e = loss_sum(&L, s)) != cudaSuccess) return e;
    total += L;
  }
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
  if (meanLoss) *meanLoss = steps > 0 ? total / ((double)steps * batch) : 0.0;
  lastLoss = steps > 0 ? total / ((double)steps * batch) : lastLoss;
  return cudaSuccess;
}
// network output (un-scaled by G) at every cell of pair p
cudaError_t Net::forward_pair(int p, float* outHost, cudaStream_t s) {
  long long N = dims.nCells;
  cudaError_t e;
  if ((e = unpack(p, s)) != cudaSuccess) return e;
  if ((e = forward(s)) != cudaSuccess) return e;
  cudaMemsetAsync(outbuf, 0, sizeof(float) * N, s);
  long long n = (long long)lv[0].ntiles * 1024;
  k_head_out<<<gridv(n, 256), 256, 0, s>>>(lv[0], tiles[0], counts, db[0], params + headOff, outbuf);
  if ((e = cudaMemcpyAsync(outHost, outbuf, sizeof(float) * N, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
  return cudaStreamSynchronize(s);
}
cudaError_t Net::grad_pair(int p, float* gradHost, double* loss, cudaStream_t s) {
  cudaError_t e;
  if (!(gain > 0) && (e = set_gain(1.0, s)) != cudaSuccess) return e;
  cudaMemsetAsync(grads, 0, sizeof(float) * nparams, s);
  cudaMemsetAsync(scal + 2, 0, sizeof(double), s);
  if ((e = sample_grad(p, s)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(gradHost, grads, sizeof(float) * nparams, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
  if (loss && (e = cudaMemcpyAsync(loss, scal + 2, sizeof(double), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
  return cudaStreamSynchronize(s);
}
// dense copies of pair p: its tiles' voxels, zero (air) elsewhere
cudaError_t Net::get_pair(int p, float* r0nHost, uint8_t* typeHost, float* targetHost, cudaStream_t s) {
  const long long N = dims.nCells;
  cudaError_t e;
  cudaMemsetAsync(r0n, 0, sizeof(float) * N, s);
  cudaMemsetAsync(typebuf, WS_AIR, (size_t)N, s);
  cudaMemsetAsync(tbuf, 0, sizeof(float) * N, s);
  if ((e = unpack(p, s)) != cudaSuccess) return e;
  if (r0nHost && (e = cudaMemcpyAsync(r0nHost, r0n, sizeof(float) * N, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
  if (typeHost && (e = cudaMemcpyAsync(typeHost, typebuf, (size_t)N, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
  if (targetHost && (e = cudaMemcpyAsync(targetHost, tbuf, sizeof(float) * N, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
  return cudaStreamSynchronize(s);
}
// a pair from dense host arrays (sigma 1): stored over the tiles its fluid cells make active
cudaError_t Net::put_pair(const float* r0nHost, const uint8_t* typeHost, const float* targetHost, cudaStream_t s) {
  const long long N = dims.nCells;
  cudaError_t e;
  if ((e = cudaMemcpyAsync(r0n, r0nHost, sizeof(float) * N, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(typebuf, typeHost, (size_t)N, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(tbuf, targetHost, sizeof(float) * N, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
  if (pairCap <= 0 && (e = reserve_pairs(1, typebuf, s)) != cudaSuccess) return e;
  const int slot = pairsStored % pairCap;
  const size_t V = (size_t)tileCap * 1024;
  if ((e = activity(typebuf, s)) != cudaSuccess) return e;
  int c[2];
  if ((e = cudaMemcpyAsync(&c[0], counts, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(&c[1], counts + kMaxLevels, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
  if (c[0] > tileCap) return cudaErrorInvalidValue;
  double t2 = 0;
  for (long long i = 0; i < N; i++) if (typeHost[i] == WS_FLUID) t2 += (double)targetHost[i] * targetHost[i];
  const double sc[2] = { 1.0, t2 };
  k_pair_pack<<<gridv((long long)c[0] * 1024, 256), 256, 0, s>>>(lv[0], tiles[0], counts, tileCap, r0n, typebuf, tbuf,
                                                                pr0n + V * slot, ptype + V * slot, ptarget + V * slot,
                                                                ptiles + (size_t)tileCap * slot);
  if ((e = cudaMemcpyAsync(pmeta + 2 * slot, c, sizeof(c), cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(pscal + 2 * slot, sc, sizeof(sc), cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
  pairsStored++;
  return cudaSuccess;
}

}  // namespace unet
