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
struct Levels { Level l[kLevels]; uint8_t* act[kLevels]; int* tiles[kLevels]; int* count; };
// one CTA: coarser activity from the finer, then the compacted tile lists
__global__ void k_tile_lists(Levels Ls) {
  __shared__ int wsum[32], carry;
  for (int lv = 0; lv < kLevels; lv++) {
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
__global__ void k_residual0(Dims d, const float* __restrict__ q, const float* __restrict__ rhs,
                            const uint8_t* __restrict__ diag8, const uint8_t* __restrict__ type,
                            float* __restrict__ r0, double* __restrict__ partials) {
  __shared__ double ws[32];
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double rr = 0;
  if (c < d.nCells) {
    float r = 0.f;
    if (type[c] == WS_FLUID) {
      int i, j, k; cell_ijk(d, c, i, j, k);
      long long nx = d.nx, nxy = (long long)d.nx * d.ny;
      double s = 0;
      if (i > 0) s += q[c - 1];
      if (i < d.nx - 1) s += q[c + 1];
      if (j > 0) s += q[c - nx];
      if (j < d.ny - 1) s += q[c + nx];
      if (k > 0) s += q[c - nxy];
      if (k < d.nz - 1) s += q[c + nxy];
      double rd = (double)rhs[c] + s - (double)diag8[c] * (double)q[c];
      rr = rd * rd;
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
__global__ void k_scale(float* __restrict__ r0, long long n, const double* sigma) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c < n) r0[c] = (float)((double)r0[c] / *sigma);
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

const LayerSpec kLayers[kNumLayers] = {
  // name, level, c0 (upsampled), c1, cout
  {"e0a", 0, 0, 16, 16}, {"e0b", 0, 0, 16, 16},
  {"e1a", 1, 0, 16, 32}, {"e1b", 1, 0, 32, 32},
  {"ba", 2, 0, 32, 64},  {"bb", 2, 0, 64, 64},
  {"d1a", 1, 64, 32, 32}, {"d1b", 1, 0, 32, 32},
  {"d0a", 0, 32, 16, 16}, {"d0b", 0, 0, 16, 16},
};

long long Net::layer_weights(int l) { return 27LL * (kLayers[l].c0 + kLayers[l].c1) * kLayers[l].cout; }

cudaError_t Net::create(const Dims& d) {
  cudaError_t e;
  dims = d;
  int nx = d.nx, ny = d.ny, nz = d.nz;
  for (int l = 0; l < kLevels; l++) {
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
  if ((e = cudaMalloc(&counts, sizeof(int) * 4)) != cudaSuccess) return e;   // 3 tile counts + fluid count
  if ((e = cudaMemset(counts, 0, sizeof(int) * 4)) != cudaSuccess) return e;
  // parameters
  nparams = 0;
  for (int l = 0; l < kNumLayers; l++) { woff[l] = nparams; nparams += layer_weights(l); boff[l] = nparams; nparams += kLayers[l].cout; }
  headOff = nparams; nparams += 17;
  if ((e = cudaMalloc(&params, sizeof(float) * nparams)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&grads, sizeof(float) * nparams)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&adm, sizeof(float) * nparams)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&adv, sizeof(float) * nparams)) != cudaSuccess) return e;
  for (int l = 0; l < kNumLayers; l++) {
    if ((e = cudaMalloc(&fw[l], sizeof(bf16) * layer_weights(l))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&bw[l], sizeof(bf16) * layer_weights(l))) != cudaSuccess) return e;
  }
  // activations and gradients (NDHWC bf16, dense per level)
  auto A = [&](bf16** p, int l, int ch) -> cudaError_t {
    cudaError_t r = cudaMalloc(p, sizeof(bf16) * lv[l].nvox * ch);
    if (r == cudaSuccess) r = cudaMemset(*p, 0, sizeof(bf16) * lv[l].nvox * ch);
    return r;
  };
  bf16** acts[] = { &x, &e0a, &s0, &d0a, &h, &gh, &gd0a, &gs0a, &gs0, &ge0a };
  for (bf16** p : acts) if ((e = A(p, 0, 16)) != cudaSuccess) return e;
  if ((e = A(&gup1, 0, 32)) != cudaSuccess) return e;
  bf16** l1_16[] = { &p1, &gp1 };
  for (bf16** p : l1_16) if ((e = A(p, 1, 16)) != cudaSuccess) return e;
  bf16** l1_32[] = { &e1a, &s1, &d1a, &d1b, &gd1b, &gd1a, &gs1a, &gs1, &ge1a };
  for (bf16** p : l1_32) if ((e = A(p, 1, 32)) != cudaSuccess) return e;
  if ((e = A(&gup2, 1, 64)) != cudaSuccess) return e;
  if ((e = A(&p2, 2, 32)) != cudaSuccess) return e;
  if ((e = A(&gp2, 2, 32)) != cudaSuccess) return e;
  bf16** l2_64[] = { &ba, &bb, &gbb, &gba };
  for (bf16** p : l2_64) if ((e = A(p, 2, 64)) != cudaSuccess) return e;
  long long N = d.nCells;
  nPartials = (int)grid1(N, 256);
  if ((e = cudaMalloc(&partials, sizeof(double) * nPartials)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&scal, sizeof(double) * 8)) != cudaSuccess) return e;   // sigma, gain, loss, t2
  if ((e = cudaMemset(scal, 0, sizeof(double) * 8)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&r0n, sizeof(float) * N)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&qprev, sizeof(float) * N)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&tscaled, sizeof(float) * N)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&outbuf, sizeof(float) * N)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&err, sizeof(int))) != cudaSuccess) return e;
  if ((e = cudaMemset(err, 0, sizeof(int))) != cudaSuccess) return e;
  return conv3_init();
}

void Net::destroy() {
  void* bufs[] = { counts, params, grads, adm, adv, x, e0a, s0, d0a, h, gh, gd0a, gs0a, gs0, ge0a, gup1, p1, gp1,
                   e1a, s1, d1a, d1b, gd1b, gd1a, gs1a, gs1, ge1a, gup2, p2, gp2, ba, bb, gbb, gba,
                   partials, scal, r0n, qprev, tscaled, outbuf, err, pr0n, ptype, ptarget, pscal };
  for (void* b : bufs) if (b) cudaFree(b);
  for (int l = 0; l < kLevels; l++) { if (act[l]) cudaFree(act[l]); if (tiles[l]) cudaFree(tiles[l]); }
  for (int l = 0; l < kNumLayers; l++) { if (fw[l]) cudaFree(fw[l]); if (bw[l]) cudaFree(bw[l]); }
}

cudaError_t Net::init_weights(uint32_t seed, cudaStream_t s) {
  std::vector<float> P((size_t)nparams, 0.f);
  HostRng rng(seed);
  for (int l = 0; l < kNumLayers; l++) {
    int cin = kLayers[l].c0 + kLayers[l].c1;
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
  for (int l = 0; l < kNumLayers; l++) {
    int n = (int)layer_weights(l);
    k_pack<<<grid1(n, 256), 256, 0, s>>>(params + woff[l], kLayers[l].c0 + kLayers[l].c1, kLayers[l].cout, fw[l], bw[l]);
  }
  return cudaGetLastError();
}

// tile activity of all levels from cell types; counts[3] = fluid cells
cudaError_t Net::activity(const uint8_t* type, cudaStream_t s) {
  cudaMemsetAsync(counts + 3, 0, sizeof(int), s);
  k_activity0<<<lv[0].ntiles, 256, 0, s>>>(lv[0], type, act[0], counts + 3);
  Levels Ls;
  for (int l = 0; l < kLevels; l++) { Ls.l[l] = lv[l]; Ls.act[l] = act[l]; Ls.tiles[l] = tiles[l]; }
  Ls.count = counts;
  k_tile_lists<<<1, 1024, 0, s>>>(Ls);
  return cudaGetLastError();
}

cudaError_t Net::conv(int l, const bf16* src0, const bf16* src1, bf16* out, cudaStream_t s) {
  const LayerSpec& S = kLayers[l];
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
  const LayerSpec& S = kLayers[l];
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
  const LayerSpec& S = kLayers[l];
  const Level& L = lv[S.level];
  ConvArgs a{};
  a.nx = L.nx; a.ny = L.ny; a.nz = L.nz; a.ntx = L.ntx; a.nty = L.nty; a.ntz = L.ntz;
  a.tiles = tiles[S.level]; a.nTiles = counts + S.level; a.active = act[S.level];
  a.src0 = src0; a.c0 = S.c0; a.up0 = S.c0 > 0; a.src1 = src1; a.c1 = S.c1; a.err = err;
  const int cin = S.c0 + S.c1;
  return launch_dw_tc(a, dz, S.cout, grads + woff[l], grads + boff[l], L.ntiles * (cin / 16), s);
}

cudaError_t Net::pool(int fineLevel, const bf16* fine, bf16* coarse, int ch, cudaStream_t s) {
  const Level& C = lv[fineLevel + 1];
  long long n = (long long)C.ntiles * 1024 * (ch / 8);
  k_pool<<<gridv(n, 256), 256, 0, s>>>(C, tiles[fineLevel + 1], counts + fineLevel + 1, lv[fineLevel], act[fineLevel],
                                       fine, coarse, ch);
  return cudaGetLastError();
}

// forward pass on the input already in x (activity and tile lists built)
cudaError_t Net::forward(cudaStream_t s) {
  cudaError_t e;
  if ((e = conv(0, nullptr, x, e0a, s)) != cudaSuccess) return e;
  if ((e = conv(1, nullptr, e0a, s0, s)) != cudaSuccess) return e;
  if ((e = pool(0, s0, p1, 16, s)) != cudaSuccess) return e;
  if ((e = conv(2, nullptr, p1, e1a, s)) != cudaSuccess) return e;
  if ((e = conv(3, nullptr, e1a, s1, s)) != cudaSuccess) return e;
  if ((e = pool(1, s1, p2, 32, s)) != cudaSuccess) return e;
  if ((e = conv(4, nullptr, p2, ba, s)) != cudaSuccess) return e;
  if ((e = conv(5, nullptr, ba, bb, s)) != cudaSuccess) return e;
  if ((e = conv(6, bb, s1, d1a, s)) != cudaSuccess) return e;
  if ((e = conv(7, nullptr, d1a, d1b, s)) != cudaSuccess) return e;
  if ((e = conv(8, d1b, s0, d0a, s)) != cudaSuccess) return e;
  return conv(9, nullptr, d0a, h, s);
}

// backward pass from the head gradient in gh; accumulates into grads
cudaError_t Net::backward(cudaStream_t s) {
  cudaError_t e;
  auto upb = [&](int coarseLevel, const bf16* dup, const bf16* a, bf16* out, int ch) {
    const Level& C = lv[coarseLevel];
    long long n = (long long)C.ntiles * 1024 * (ch / 8);
    k_up_bwd<<<gridv(n, 256), 256, 0, s>>>(C, tiles[coarseLevel], counts + coarseLevel, lv[coarseLevel - 1],
                                           act[coarseLevel - 1], dup, a, out, ch);
    return cudaGetLastError();
  };
  auto pba = [&](int fineLevel, const bf16* dskip, const bf16* dpool, const bf16* sAct, bf16* out, int ch) {
    const Level& F = lv[fineLevel];
    long long n = (long long)F.ntiles * 1024 * (ch / 8);
    k_pool_bwd_add<<<gridv(n, 256), 256, 0, s>>>(F, tiles[fineLevel], counts + fineLevel, lv[fineLevel + 1],
                                                 dskip, dpool, sAct, out, ch);
    return cudaGetLastError();
  };
  if ((e = dw(9, nullptr, d0a, gh, s)) != cudaSuccess) return e;
  if ((e = conv_bwd(9, gh, d0a, gd0a, nullptr, s)) != cudaSuccess) return e;
  if ((e = dw(8, d1b, s0, gd0a, s)) != cudaSuccess) return e;
  if ((e = conv_bwd(8, gd0a, nullptr, gup1, gs0a, s)) != cudaSuccess) return e;
  if ((e = upb(1, gup1, d1b, gd1b, 32)) != cudaSuccess) return e;
  if ((e = dw(7, nullptr, d1a, gd1b, s)) != cudaSuccess) return e;
  if ((e = conv_bwd(7, gd1b, d1a, gd1a, nullptr, s)) != cudaSuccess) return e;
  if ((e = dw(6, bb, s1, gd1a, s)) != cudaSuccess) return e;
  if ((e = conv_bwd(6, gd1a, nullptr, gup2, gs1a, s)) != cudaSuccess) return e;
  if ((e = upb(2, gup2, bb, gbb, 64)) != cudaSuccess) return e;
  if ((e = dw(5, nullptr, ba, gbb, s)) != cudaSuccess) return e;
  if ((e = conv_bwd(5, gbb, ba, gba, nullptr, s)) != cudaSuccess) return e;
  if ((e = dw(4, nullptr, p2, gba, s)) != cudaSuccess) return e;
  if ((e = conv_bwd(4, gba, nullptr, gp2, nullptr, s)) != cudaSuccess) return e;
  if ((e = pba(1, gs1a, gp2, s1, gs1, 32)) != cudaSuccess) return e;
  if ((e = dw(3, nullptr, e1a, gs1, s)) != cudaSuccess) return e;
  if ((e = conv_bwd(3, gs1, e1a, ge1a, nullptr, s)) != cudaSuccess) return e;
  if ((e = dw(2, nullptr, p1, ge1a, s)) != cudaSuccess) return e;
  if ((e = conv_bwd(2, ge1a, nullptr, gp1, nullptr, s)) != cudaSuccess) return e;
  if ((e = pba(0, gs0a, gp1, s0, gs0, 16)) != cudaSuccess) return e;
  if ((e = dw(1, nullptr, e0a, gs0, s)) != cudaSuccess) return e;
  if ((e = conv_bwd(1, gs0, e0a, ge0a, nullptr, s)) != cudaSuccess) return e;
  return dw(0, nullptr, x, ge0a, s);
}

// input from normalised residual + cell types; builds activity first
cudaError_t Net::prepare(const float* r0nIn, const uint8_t* type, cudaStream_t s) {
  cudaError_t e;
  if ((e = activity(type, s)) != cudaSuccess) return e;
  long long n = (long long)lv[0].ntiles * 1024;
  k_input<<<gridv(n, 256), 256, 0, s>>>(lv[0], tiles[0], counts, r0nIn, type, x, nullptr);
  return cudaGetLastError();
}
// r0 / sigma of the current pressure setup into dst, sigma into sig
cudaError_t Net::residual(const float* q, const float* rhs, const uint8_t* diag8, const uint8_t* type,
                          float* dst, double* sig, cudaStream_t s, bool scale) {
  long long N = dims.nCells;
  k_residual0<<<nPartials, 256, 0, s>>>(dims, q, rhs, diag8, type, dst, partials);
  k_sigma<<<1, 1024, 0, s>>>(partials, nPartials, counts + 3, sig);
  if (scale) k_scale<<<grid1(N, 256), 256, 0, s>>>(dst, N, sig);
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
  k_head_apply<<<gridv(n, 256), 256, 0, s>>>(lv[0], tiles[0], counts, h, params + headOff, type, scal + 0, scal + 1, q);
  return cudaGetLastError();
}

// ---- training pairs
cudaError_t Net::reserve_pairs(int capacity) {
  if (capacity <= pairCap) return cudaSuccess;
  long long N = dims.nCells;
  float *a = nullptr, *c = nullptr; uint8_t* b = nullptr; double* sc = nullptr;
  cudaError_t e;
  if ((e = cudaMalloc(&a, sizeof(float) * N * capacity)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&b, (size_t)N * capacity)) != cudaSuccess) { cudaFree(a); return e; }
  if ((e = cudaMalloc(&c, sizeof(float) * N * capacity)) != cudaSuccess) { cudaFree(a); cudaFree(b); return e; }
  if ((e = cudaMalloc(&sc, sizeof(double) * 2 * capacity)) != cudaSuccess) { cudaFree(a); cudaFree(b); cudaFree(c); return e; }
  cudaMemset(sc, 0, sizeof(double) * 2 * capacity);
  if (pairCap > 0 && pairsStored > 0) {   // keep the stored pairs
    int keep = std::min(pairsStored, pairCap);
    cudaMemcpy(a, pr0n, sizeof(float) * N * keep, cudaMemcpyDeviceToDevice);
    cudaMemcpy(b, ptype, (size_t)N * keep, cudaMemcpyDeviceToDevice);
    cudaMemcpy(c, ptarget, sizeof(float) * N * keep, cudaMemcpyDeviceToDevice);
    cudaMemcpy(sc, pscal, sizeof(double) * 2 * keep, cudaMemcpyDeviceToDevice);
  }
  cudaFree(pr0n); cudaFree(ptype); cudaFree(ptarget); cudaFree(pscal);
  pr0n = a; ptype = b; ptarget = c; pscal = sc; pairCap = capacity;
  return cudaSuccess;
}
// before the solve: slot <- (r0 / sigma, types), q_prev saved
cudaError_t Net::collect_pre(const float* q, const float* rhs, const uint8_t* diag8, const uint8_t* type, cudaStream_t s) {
  if (pairCap <= 0) return cudaSuccess;
  long long N = dims.nCells;
  int slot = pairsStored % pairCap;
  cudaError_t e;
  if ((e = activity(type, s)) != cudaSuccess) return e;
  if ((e = residual(q, rhs, diag8, type, pr0n + N * slot, pscal + 2 * slot, s)) != cudaSuccess) return e;
  cudaMemcpyAsync(ptype + N * slot, type, (size_t)N, cudaMemcpyDeviceToDevice, s);
  cudaMemcpyAsync(qprev, q, sizeof(float) * N, cudaMemcpyDeviceToDevice, s);
  return cudaGetLastError();
}
// after the solve: target = (q - q_prev) / sigma
cudaError_t Net::collect_post(const float* q, cudaStream_t s) {
  if (pairCap <= 0) return cudaSuccess;
  long long N = dims.nCells;
  int slot = pairsStored % pairCap;
  cudaMemsetAsync(pscal + 2 * slot + 1, 0, sizeof(double), s);
  k_pair_target<<<grid1(N, 256), 256, 0, s>>>(N, q, qprev, ptype + N * slot, pscal + 2 * slot, ptarget + N * slot,
                                             pscal + 2 * slot + 1);
  pairsStored++;
  return cudaGetLastError();
}

// gain G = RMS of the stored targets over fluid cells (set once, before the first training step)
cudaError_t Net::set_gain_from_pairs(cudaStream_t s) {
  int n = std::min(pairsStored, pairCap);
  if (n <= 0) return cudaErrorInvalidValue;
  std::vector<double> sc((size_t)2 * n);
  cudaError_t e = cudaMemcpyAsync(sc.data(), pscal, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
  // fluid counts: per pair, from the activity pass (host loop over the pairs)
  double t2 = 0, cnt = 0;
  long long N = dims.nCells;
  for (int p = 0; p < n; p++) {
    if ((e = activity(ptype + N * p, s)) != cudaSuccess) return e;
    int c4[4];
    if ((e = cudaMemcpyAsync(c4, counts, sizeof(int) * 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
    t2 += sc[(size_t)2 * p + 1]; cnt += c4[3];
  }
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
  if ((e = prepare(pr0n + N * p, ptype + N * p, s)) != cudaSuccess) return e;
  if ((e = forward(s)) != cudaSuccess) return e;
  k_scale_copy<<<grid1(N, 256), 256, 0, s>>>(ptarget + N * p, tscaled, N, (float)(1.0 / gain));
  long long n = (long long)lv[0].ntiles * 1024;
  k_head_train<<<gridv(n, 256), 256, 0, s>>>(lv[0], tiles[0], counts, h, params + headOff, ptype + N * p, tscaled,
                                             counts + 3, gh, grads + headOff, scal + 2);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  return backward(s);
}
// zero the gradients and the loss, then add the gradients of `samples`
// pairs drawn with a seeded generator (no parameter update)
cudaError_t Net::accumulate(int samples, uint32_t seed, cudaStream_t s) {
  int n = std::min(pairsStored, pairCap);
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
  int n = std::min(pairsStored, pairCap);
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
  if ((e = prepare(pr0n + N * p, ptype + N * p, s)) != cudaSuccess) return e;
  if ((e = forward(s)) != cudaSuccess) return e;
  cudaMemsetAsync(outbuf, 0, sizeof(float) * N, s);
  long long n = (long long)lv[0].ntiles * 1024;
  k_head_out<<<gridv(n, 256), 256, 0, s>>>(lv[0], tiles[0], counts, h, params + headOff, outbuf);
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

}  // namespace unet
