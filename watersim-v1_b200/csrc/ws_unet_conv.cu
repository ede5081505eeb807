// ws_unet_conv.cu — 3x3x3 convolution of the warm-start U-Net as an
// implicit GEMM on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// One CTA computes a sub-tile of 8 (x) x 16 (y) x ZT (z) output voxels of one
// active tile. For each 16-channel slice of the input it stages, in shared
// memory, the (8+2) x (16+2) x (ZT+2) halo of that slice (two 8-channel
// chunks, voxel-major, 16 bytes per voxel per chunk) and the slice's weights
// for all 27 taps. One elected thread then issues, for every output plane z
// and tap (dz, dy, dx), one tcgen05.mma of M = 128 (the 8 x 16 voxels of the
// plane), N = cout, K = 16 (the channel slice), BF16 inputs, FP32
// accumulator in tensor memory. The A operand of a tap is the halo shifted by
// (dz, dy, dx): with the no-swizzle K-major layout each 8-row core matrix is
// the 8 x-consecutive voxels of one y-row (128 contiguous bytes), the stride
// between core matrices along M is one halo row (160 bytes) and the stride
// between the two K chunks is one halo chunk, so a shift only moves the
// descriptor's start address. Inactive neighbour tiles and voxels outside
// the grid are staged as zeros. The epilogue reads the accumulators with
// tcgen05.ld (each warp its 32-lane quarter), adds bias and ReLU (forward)
// or applies a ReLU mask (backward data), and stores BF16 NDHWC.
//
// Every mbarrier wait is bounded; on a timeout the CTA latches
// WS_DERR_TIMEOUT, waits once more (bounded) for its MMAs, frees its tensor
// memory and returns.
#include "ws_unet.cuh"
#include <algorithm>

namespace unet {

static constexpr long long kWaitLimit = 1LL << 24;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor, no swizzle: start, leading (K-chunk) and
// stride (8-row group) byte offsets in 16-byte units, descriptor version 1
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}
// instruction descriptor of kind::f16: D f32, A bf16, B bf16, both K-major, M = 128
__host__ __device__ constexpr uint32_t idesc_bf16_m128(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}
__device__ __forceinline__ void mma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
               "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
               :: "r"(d), "l"(a), "l"(b), "r"(idesc), "r"(acc) : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :: "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
               "selp.u32 %0, 1, 0, p;\n\t}\n" : "=r"(done) : "r"(smem_u32(bar)), "r"(parity) : "memory");
  return done != 0;
}
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (long long n = 0; n < kWaitLimit; n++)
    if (mbar_try(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                 "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Output planes per work item: eight (a whole tile) up to 32 channels; two
// from 48 to 128 channels, which run on the coarse levels, where a tile per
// item would leave most SMs idle (the 32^3 level of a 128^3 grid has 32
// tiles) and each CTA would walk four or more input slices in turn.
template <int COUT> struct ConvShape {
  static constexpr int ZT = COUT <= 32 ? 8 : COUT <= 128 ? 2 : 1;
  static constexpr int HX = kTX + 2, HY = kTY + 2, HZ = ZT + 2;
  static constexpr int HV = HX * HY * HZ;           // halo voxels
  static constexpr int KSTR = HV * 16;              // bytes of one 8-channel halo chunk
  static constexpr int WCH = 27 * 2 * COUT * 16;    // bytes of one 16-channel weight slice
  static constexpr int NCOL = ZT * COUT;
  static constexpr int TCOLS = NCOL <= 32 ? 32 : NCOL <= 64 ? 64 : NCOL <= 128 ? 128 : NCOL <= 256 ? 256 : 512;
  // shared memory per CTA, padded so that the CTAs one SM can hold never
  // ask for more than the 512 tensor-memory columns together (233472 bytes
  // of shared memory per SM, 1 KB of it reserved per CTA)
  static constexpr int MAXCTA = 512 / TCOLS;
  static constexpr int SMEM_MIN = 233472 / (MAXCTA + 1) + 1;
  static constexpr int SMEM = 2 * KSTR + WCH > SMEM_MIN ? 2 * KSTR + WCH : SMEM_MIN;
};

// 16-byte asynchronous global -> shared copy; src_size 0 writes zeros
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t src_size) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" :: "r"(dst), "l"(src), "r"(src_size) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// queue the copies of one 16-channel slice of the halo of sub-tile (X0, Y0, Z0).
// The activity of the (up to) 3x3x3 tiles the halo touches is read once into
// shared memory, so no copy waits on a global load of its own.
template <int COUT>
__device__ __forceinline__ void stage_halo(const ConvArgs& a, int X0, int Y0, int Z0, int kk, uint32_t hbase,
                                           uint8_t* s_act) {
  using S = ConvShape<COUT>;
  constexpr int HX = S::HX, HY = S::HY, HV = S::HV, KSTR = S::KSTR;
  const int tx0 = X0 / kTX - 1, ty0 = Y0 / kTY - 1, tz0 = (Z0 + kTZ - 1) / kTZ - 1;   // tile of the halo's low corner
  if (threadIdx.x < 27) {
    const int t = threadIdx.x, tx = tx0 + t % 3, ty = ty0 + (t / 3) % 3, tz = tz0 + t / 9;
    s_act[t] = (tx >= 0 && ty >= 0 && tz >= 0 && tx < a.ntx && ty < a.nty && tz < a.ntz)
                   ? a.active[(tz * a.nty + ty) * a.ntx + tx] : (uint8_t)0;
  }
  __syncthreads();
  const int cnx = (a.nx + 1) >> 1, cny = (a.ny + 1) >> 1;
  // one voxel per thread and pass, both 8-channel chunks of the slice (the
  // channel splits c0 are multiples of 16, so both come from one source)
  for (int hv = threadIdx.x; hv < HV; hv += blockDim.x) {
    const int hx = hv % HX, t2 = hv / HX, hy = t2 % HY, hz = t2 / HY;
    const int gx = X0 - 1 + hx, gy = Y0 - 1 + hy, gz = Z0 - 1 + hz;
    const bf16* p = a.src1 ? a.src1 : a.src0;             // any valid address when nothing is read
    uint32_t n = 0;
    if (gx >= 0 && gy >= 0 && gz >= 0 && gx < a.nx && gy < a.ny && gz < a.nz &&
        s_act[((gz / kTZ - tz0) * 3 + (gy / kTY - ty0)) * 3 + (gx / kTX - tx0)]) {
      const int c = kk * 16;
      if (c < a.c0) {
        p = a.up0 ? a.src0 + ((size_t)((gz >> 1) * cny + (gy >> 1)) * cnx + (gx >> 1)) * a.c0 + c
                  : a.src0 + ((size_t)(gz * a.ny + gy) * a.nx + gx) * a.c0 + c;
      } else {
        p = a.src1 + ((size_t)(gz * a.ny + gy) * a.nx + gx) * a.c1 + (c - a.c0);
      }
      n = 16;
    }
    cp_async16(hbase + (uint32_t)(hv * 16), p, n);
    cp_async16(hbase + (uint32_t)(KSTR + hv * 16), p + 8, n);
  }
}
template <int COUT>
__device__ __forceinline__ void stage_weights(const ConvArgs& a, int kk, uint32_t wbase) {
  constexpr int WCH = ConvShape<COUT>::WCH;
  const char* src = reinterpret_cast<const char*>(a.w) + (size_t)kk * WCH;
  for (int i = threadIdx.x; i < WCH / 16; i += blockDim.x) cp_async16(wbase + (uint32_t)(i * 16), src + (size_t)i * 16, 16);
}

// Persistent over the work items (active tile x z sub-tile): tensor memory
// is allocated once per CTA; weights stay resident when the input has a
// single 16-channel slice; the next item's first slice is fetched while
// the current item's accumulators are drained.
template <int COUT>
__global__ void __launch_bounds__(256) k_conv3(ConvArgs a) {
  using S = ConvShape<COUT>;
  constexpr int ZT = S::ZT, HX = S::HX, HY = S::HY, KSTR = S::KSTR;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t s_tmem;
  __shared__ int s_abort;
  __shared__ uint8_t s_act[27];

  constexpr int sub = kTZ / ZT;
  const int nItems = *a.nTiles * sub;
  if ((int)blockIdx.x >= nItems) return;            // uniform over the CTA
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t hbase = smem_u32(smem), wbase = hbase + 2 * KSTR;
  const int cin = a.c0 + a.c1, nslices = cin >> 4;
  const bool wres = nslices == 1;                   // weights loaded once

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(&s_tmem)), "r"((uint32_t)S::TCOLS) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 32) { mbar_init(&mbar, 1); s_abort = 0; }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = s_tmem;
  constexpr uint32_t idesc = idesc_bf16_m128(COUT);
  // N = 2 and 3 COUT (two or three z taps); with ZT = 2 at most two z taps meet one plane
  constexpr uint32_t idesc2 = idesc_bf16_m128(2 * COUT);
  constexpr uint32_t idesc3 = idesc_bf16_m128((ZT >= 3 ? 3 : 2) * COUT);
  static_assert((ZT >= 3 ? 3 : ZT) * COUT <= 256 && COUT % 16 == 0, "MMA N out of range");
  uint32_t phase = 0;
  bool pending = false;

  auto origin = [&](int item, int& X0, int& Y0, int& Z0) {
    const int tile = a.tiles[item / sub];
    const int tx = tile % a.ntx, ty = (tile / a.ntx) % a.nty, tz = tile / (a.ntx * a.nty);
    X0 = tx * kTX; Y0 = ty * kTY; Z0 = tz * kTZ + (item % sub) * ZT;
  };
  int X0, Y0, Z0;
  origin(blockIdx.x, X0, Y0, Z0);
  stage_halo<COUT>(a, X0, Y0, Z0, 0, hbase, s_act);
  stage_weights<COUT>(a, 0, wbase);
  for (int item = blockIdx.x; item < nItems; item += gridDim.x) {
    for (int kk = 0; kk < nslices; kk++) {
      cp_async_wait_all();
      fence_proxy_async();                           // generic-proxy writes -> tensor-core reads
      __syncthreads();
      if (threadIdx.x == 0) {
        fence_after();
        // Per in-plane tap g = (dy, dx), halo plane p feeds output planes
        // p - dz for dz = 0..2: one MMA with the B rows of those z taps side
        // by side along N (k_pack orders them dz = 2, 1, 0) writes the
        // accumulators of planes p - dzhi .. p - dzlo, which are adjacent in
        // tensor memory. Each A tile is then read once per (g, p) instead of
        // once per (g, dz, z). The first tap group initialises every
        // accumulator plane by plane (dz = 0 first), the later groups only
        // accumulate. Descriptors are base descriptors plus 16-byte offsets
        // in the start-address field.
        const uint64_t ad0 = smem_desc(hbase, KSTR, HX * 16), bd0 = smem_desc(wbase, 3 * COUT * 16, 128);
        constexpr int GB = 6 * COUT;                 // 16-byte units of one tap group (2 K halves x 3 z taps)
#pragma unroll
        for (int z = 0; z < ZT; z++)
#pragma unroll
          for (int dz = 0; dz < 3; dz++)
            mma_bf16(tmem + (uint32_t)(z * COUT), ad0 + (uint64_t)((z + dz) * HY * HX),
                     bd0 + (uint64_t)((2 - dz) * COUT), idesc, (kk | dz) != 0);
#pragma unroll 1
        for (int g = 1; g < 9; g++) {
          const int dy = g / 3, dx = g % 3;
          const uint64_t ag = ad0 + (uint64_t)(dy * HX + dx), bg = bd0 + (uint64_t)(g * GB);
#pragma unroll
          for (int p = 0; p < ZT + 2; p++) {
            const int dzlo = p > ZT - 1 ? p - (ZT - 1) : 0, dzhi = p < 2 ? p : 2;
            const uint32_t id = dzhi - dzlo == 0 ? idesc : dzhi - dzlo == 1 ? idesc2 : idesc3;
            mma_bf16(tmem + (uint32_t)((p - dzhi) * COUT), ag + (uint64_t)(p * HY * HX),
                     bg + (uint64_t)((2 - dzhi) * COUT), id, 1u);
          }
        }
        mma_commit(&mbar);
      }
      pending = true;
      const bool ok = mbar_wait(&mbar, phase);       // the staged operands are free again
      if (!ok) { s_abort = 1; atomicOr(a.err, WS_DERR_TIMEOUT); }
      __syncthreads();
      if (s_abort) break;
      pending = false;
      phase ^= 1u;
      if (kk + 1 < nslices) {
        stage_halo<COUT>(a, X0, Y0, Z0, kk + 1, hbase, s_act);
        stage_weights<COUT>(a, kk + 1, wbase);
      }
    }
    if (s_abort) break;
    // fetch the next item's first slice while this item's accumulators drain
    const int cX = X0, cY = Y0, cZ = Z0;
    const int next = item + gridDim.x;
    if (next < nItems) {
      origin(next, X0, Y0, Z0);
      stage_halo<COUT>(a, X0, Y0, Z0, 0, hbase, s_act);
      if (!wres) stage_weights<COUT>(a, 0, wbase);
    }
    fence_after();
    {
      const int q = warp & 3;                        // tensor-memory lane quarter of this warp
      const int m = q * 32 + lane;                   // accumulator row = voxel of the plane
      const int gx = cX + (m & 7), gy = cY + (m >> 3);
#pragma unroll 1
      for (int cg = 0; cg < COUT / 16; cg++) {
        const int c = cg * 16;
        float bias[16];                              // this channel group's bias, once for all planes
#pragma unroll
        for (int i = 0; i < 16; i++) bias[i] = a.mode == 0 ? __ldg(a.bias + c + i) : 0.f;
        for (int z = warp >> 2; z < ZT; z += 2) {
          const int gz = cZ + z;
          const bool in = gx < a.nx && gy < a.ny && gz < a.nz;
          const size_t vox = ((size_t)gz * a.ny + gy) * a.nx + gx;
          uint32_t r[16];
          tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(z * COUT + cg * 16), r);
          if (!in) continue;
          float v[16];
#pragma unroll
          for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
          if (a.mode == 0) {
#pragma unroll
            for (int i = 0; i < 16; i++) v[i] = fmaxf(v[i] + bias[i], 0.f);
          } else if (a.mask) {
            const uint4* mp = reinterpret_cast<const uint4*>(a.mask + vox * COUT + c);
            uint4 mk[2] = { __ldg(mp), __ldg(mp + 1) };
            const bf16* mb = reinterpret_cast<const bf16*>(mk);
#pragma unroll
            for (int i = 0; i < 16; i++) if (!(__bfloat162float(mb[i]) > 0.f)) v[i] = 0.f;
          }
          uint4 o[2];
          __nv_bfloat162* ob = reinterpret_cast<__nv_bfloat162*>(o);
#pragma unroll
          for (int i = 0; i < 8; i++) ob[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
          uint4* dst = c < a.split
              ? reinterpret_cast<uint4*>(a.out0 + vox * a.split + c)
              : reinterpret_cast<uint4*>(a.out1 + vox * (COUT - a.split) + (c - a.split));
          dst[0] = o[0]; dst[1] = o[1];
        }
      }
    }
    fence_before();                                  // accumulators read before the next item's MMAs
  }
  if (s_abort && pending) mbar_wait(&mbar, phase);    // bounded: let the issued MMAs drain
  cp_async_wait_all();
  fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"((uint32_t)S::TCOLS) : "memory");
}

// ------------------------------------------------------------ weight gradient
// dW[co][ci][t] += sum_v X(v + off_t)[ci] dZ(v)[co] over the voxels of
// active tiles, on the tensor cores. One CTA per (active tile, 16-channel
// input slice), persistent, one per SM. Per tap t the GEMM is D[co][ci] =
// sum over voxels: A = dZ (M = 64 rows, cout <= 64 real), B = the input halo
// shifted by the tap (N = 16 channels), K = 16 voxels (two x-rows of a plane)
// per MMA. Both operands are MN-major: a core matrix is 8 channels (16
// bytes) by 8 consecutive voxels; K groups are 128 bytes apart in the staged
// dZ and one halo row (160 bytes) apart in the halo. The whole tile's dZ and
// halo are staged once; the 8 planes x 8 K steps x 27 taps = 1728 MMAs are
// issued back to back (taps innermost: 27 independent accumulators of 16
// columns) with descriptors formed by adding 16-byte offsets to two base
// descriptors, and drained once per item.
// one pass covers output channels coOff .. coOff + cout - 1 (cout <= 64) of a
// dZ with dzStride channels per voxel
struct DwTcArgs { ConvArgs src; const bf16* dz; int cout, dzStride, coOff; float* dw; float* db; };
constexpr int kDzPlane = 128 * 16;                // bytes of one plane of one 8-channel chunk of dZ
constexpr int kDzChunk = kTZ * kDzPlane;          // one 8-channel chunk of the tile's dZ
constexpr int kDwTcSmem = 2 * ConvShape<16>::KSTR + 8 * kDzChunk;
static_assert(kDwTcSmem + 1024 <= 232448, "halo and dZ of a tile fit one CTA's shared memory");
// instruction descriptor: D f32, A and B bf16, both MN-major, M = 64, N = 16.
// With M = 64 the accumulator rows 16q..16q+15 sit in tensor-memory lanes
// 32q..32q+15 (the lower half of each 32-lane subpartition).
constexpr uint32_t kIdescDw = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) |
                              ((uint32_t)(16 >> 3) << 17) | ((uint32_t)(64 >> 4) << 24);

__global__ void __launch_bounds__(256, 1) k_dw_tc(DwTcArgs A) {
  const ConvArgs& a = A.src;
  using S = ConvShape<16>;                          // ZT = 8: the whole tile's halo of one slice
  constexpr int HX = S::HX, HY = S::HY, KSTR = S::KSTR;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t s_tmem;
  __shared__ int s_abort;
  __shared__ uint8_t s_act[27];
  const int cin = a.c0 + a.c1, nsl = cin >> 4, cout = A.cout;
  const int nItems = *a.nTiles * nsl;
  if ((int)blockIdx.x >= nItems) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t hbase = smem_u32(smem), zbase = hbase + 2 * KSTR;
  unsigned char* zbuf = smem + 2 * KSTR;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" :: "r"(smem_u32(&s_tmem)), "r"(512u) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 32) { mbar_init(&mbar, 1); s_abort = 0; }
  // rows co >= cout of the A operand read zeros
  for (int i = threadIdx.x; i < 8 * kDzChunk / 16; i += blockDim.x) reinterpret_cast<uint4*>(zbuf)[i] = make_uint4(0u, 0u, 0u, 0u);
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = s_tmem;
  const uint64_t adesc0 = smem_desc(zbase, 128, kDzChunk), bdesc0 = smem_desc(hbase, HX * 16, KSTR);
  uint32_t phase = 0;
  bool pending = false;
  for (int item = blockIdx.x; item < nItems && !s_abort; item += gridDim.x) {
    const int tile = a.tiles[item / nsl], kk = item % nsl;
    const int tx = tile % a.ntx, ty = (tile / a.ntx) % a.nty, tz = tile / (a.ntx * a.nty);
    const int X0 = tx * kTX, Y0 = ty * kTY, Z0 = tz * kTZ;
    stage_halo<16>(a, X0, Y0, Z0, kk, hbase, s_act);
    for (int i = threadIdx.x; i < (cout >> 3) * kTZ * 128; i += blockDim.x) {
      const int c = i / (kTZ * 128), r = i - c * (kTZ * 128), z = r >> 7, m = r & 127;
      const int gx = X0 + (m & 7), gy = Y0 + (m >> 3), gz = Z0 + z;
      const bool in = gx < a.nx && gy < a.ny && gz < a.nz;
      const bf16* src = in ? A.dz + (((size_t)gz * a.ny + gy) * a.nx + gx) * A.dzStride + A.coOff + c * 8 : A.dz;
      cp_async16(zbase + (uint32_t)(c * kDzChunk + z * kDzPlane + m * 16), src, in ? 16u : 0u);
    }
    cp_async_wait_all();
    fence_proxy_async();
    __syncthreads();
    if (threadIdx.x == 0) {
      fence_after();
#pragma unroll 1
      for (int z = 0; z < kTZ; z++) {
#pragma unroll 1
        for (int ks = 0; ks < 8; ks++) {
          const uint64_t ad = adesc0 + (uint64_t)((z * kDzPlane + ks * 256) >> 4);
          const uint32_t rowb = (uint32_t)(z * HY + 2 * ks) * HX;       // halo row of tap (0, 0, 0), 16-byte units
#pragma unroll
          for (int t = 0; t < 27; t++) {
            const int dz = t / 9, dy = (t / 3) % 3, dx = t % 3;
            const uint64_t bd = bdesc0 + (uint64_t)(rowb + (uint32_t)((dz * HY + dy) * HX + dx));
            mma_bf16(tmem + (uint32_t)(t * 16), ad, bd, kIdescDw, (z | ks) != 0);
          }
        }
      }
      mma_commit(&mbar);
    }
    pending = true;
    float bsum = 0.f;                                // bias gradient while the MMAs run
    if (kk == 0 && (int)threadIdx.x < cout) {
      const bf16* col = reinterpret_cast<const bf16*>(zbuf + (threadIdx.x >> 3) * kDzChunk) + (threadIdx.x & 7);
      for (int m = 0; m < kTZ * 128; m++) bsum += __bfloat162float(col[m * 8]);
    }
    const bool ok = mbar_wait(&mbar, phase);
    if (!ok) { s_abort = 1; atomicOr(a.err, WS_DERR_TIMEOUT); }
    __syncthreads();
    if (s_abort) break;
    pending = false;
    phase ^= 1u;
    fence_after();
    {
      const int q = warp & 3, co = lane < 16 ? q * 16 + lane : 1 << 20;   // accumulator row of this lane
      for (int t = warp >> 2; t < 27; t += 2) {
        uint32_t r[16];
        tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(t * 16), r);
        if (co < cout) {
#pragma unroll
          for (int i = 0; i < 16; i++)
            atomicAdd(A.dw + ((size_t)(A.coOff + co) * cin + kk * 16 + i) * 27 + t, __uint_as_float(r[i]));
        }
      }
    }
    if (kk == 0 && (int)threadIdx.x < cout) atomicAdd(A.db + A.coOff + threadIdx.x, bsum);
    fence_before();
    __syncthreads();                                 // accumulators and staged operands free for the next item
  }
  if (s_abort && pending) mbar_wait(&mbar, phase);
  cp_async_wait_all();
  fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(512u) : "memory");
}
cudaError_t launch_dw_tc(const ConvArgs& src, const bf16* dz, int cout, float* dw, float* db, int maxItems,
                         cudaStream_t s) {
  if (((src.c0 + src.c1) & 15) || (cout & 7) || cout > 128) return cudaErrorInvalidValue;
  static int smCount = 0;
  if (!smCount) { int dev = 0; cudaGetDevice(&dev); cudaDeviceGetAttribute(&smCount, cudaDevAttrMultiProcessorCount, dev); }
  const unsigned grid = (unsigned)std::min(maxItems, smCount);     // one CTA per SM: 512 TMEM columns each
  if (grid == 0) return cudaSuccess;
  for (int off = 0; off < cout; off += 64) {       // the A operand holds 64 output channels per pass
    DwTcArgs A{src, dz, std::min(64, cout - off), cout, off, dw, db};
    k_dw_tc<<<grid, 256, kDwTcSmem, s>>>(A);
  }
  return cudaGetLastError();
}

template <int COUT> static cudaError_t set_smem() {
  return cudaFuncSetAttribute(k_conv3<COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, ConvShape<COUT>::SMEM);
}
cudaError_t conv3_init() {
  cudaError_t e;
  if ((e = set_smem<16>()) != cudaSuccess) return e;
  if ((e = set_smem<32>()) != cudaSuccess) return e;
  if ((e = set_smem<48>()) != cudaSuccess) return e;
  if ((e = set_smem<64>()) != cudaSuccess) return e;
  if ((e = set_smem<96>()) != cudaSuccess) return e;
  if ((e = set_smem<128>()) != cudaSuccess) return e;
  if ((e = set_smem<192>()) != cudaSuccess) return e;
  // the weight-gradient kernel holds more than half an SM's shared memory: one CTA per SM
  return cudaFuncSetAttribute(k_dw_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kDwTcSmem);
}
int conv3_zt(int cout) {
  switch (cout) {
    case 16: return ConvShape<16>::ZT; case 32: return ConvShape<32>::ZT; case 48: return ConvShape<48>::ZT;
    case 64: return ConvShape<64>::ZT; case 96: return ConvShape<96>::ZT; case 128: return ConvShape<128>::ZT;
    case 192: return ConvShape<192>::ZT; default: return 0;
  }
}
size_t conv3_smem_bytes(int cout) {
  switch (cout) {
    case 16: return ConvShape<16>::SMEM; case 32: return ConvShape<32>::SMEM; case 48: return ConvShape<48>::SMEM;
    case 64: return ConvShape<64>::SMEM; case 96: return ConvShape<96>::SMEM; case 128: return ConvShape<128>::SMEM;
    case 192: return ConvShape<192>::SMEM; default: return 0;
  }
}
cudaError_t launch_conv3(const ConvArgs& a, int cout, int maxTiles, cudaStream_t s) {
  // the halo staging takes both 8-channel chunks of a slice from one source: splits are multiples of 16
  if (((a.c0 + a.c1) & 15) || (a.c0 & 15) || a.c0 + a.c1 <= 0 || (a.split & 15)) return cudaErrorInvalidValue;
  const int zt = conv3_zt(cout);
  if (!zt) return cudaErrorInvalidValue;
  // persistent: at most the CTAs the device holds at once, never more than the work items
  static int smCount = 0;
  if (!smCount) { int dev = 0; cudaGetDevice(&dev); cudaDeviceGetAttribute(&smCount, cudaDevAttrMultiProcessorCount, dev); }
  const size_t smb = conv3_smem_bytes(cout);
  const int perSM = (int)(233472 / (smb + 1024 + 256));
  const long long items = (long long)maxTiles * (kTZ / zt);
  const dim3 grid((unsigned)std::min<long long>(items, (long long)smCount * std::max(perSM, 1)));
  if (grid.x == 0) return cudaSuccess;
  const size_t sm = conv3_smem_bytes(cout);
  switch (cout) {
    case 16: k_conv3<16><<<grid, 256, sm, s>>>(a); break;
    case 32: k_conv3<32><<<grid, 256, sm, s>>>(a); break;
    case 48: k_conv3<48><<<grid, 256, sm, s>>>(a); break;
    case 64: k_conv3<64><<<grid, 256, sm, s>>>(a); break;
    case 96: k_conv3<96><<<grid, 256, sm, s>>>(a); break;
    case 128: k_conv3<128><<<grid, 256, sm, s>>>(a); break;
    case 192: k_conv3<192><<<grid, 256, sm, s>>>(a); break;
  }
  return cudaGetLastError();
}

}  // namespace unet
