// ws_unet.cuh — the learned warm start of the pressure solve: a small 3D
// U-Net (3 or 4 levels, 16/32/64(/128) channels, 3x3x3 convolutions, BF16
// weights and activations, FP32 accumulation in tensor memory) that
// predicts the change of the pressure over one solve from the initial
// residual. The reference
// has no counterpart: its _pressureSolve (js/solver.js:1312-1410) starts SOR
// from the previous substep's q. SOR always continues from the prediction to
// the same tolerance, so the network can only change the iteration count.
//
// Sparse bricks. Every level is cut into tiles of 8 (x) x 16 (y) x 8 (z)
// voxels. A tile at level 0 is active when it holds a fluid cell; a tile at
// level l+1 is active when any of the 2x2x2 level-l tiles under it is. The
// network is defined on active tiles only: activations of inactive tiles are
// zero, and every kernel (forward, backward, the CPU oracle) reads them as
// zero. About a quarter of the 128^3 box is active for a planet ocean shell.
//
// Tensor layout: NDHWC, channels innermost, bf16, dense over the level grid
// (only active tiles are ever written or read).
#pragma once
#include "ws_internal.cuh"
#include <cuda_bf16.h>

namespace unet {

typedef __nv_bfloat16 bf16;

constexpr int kTX = 8, kTY = 16, kTZ = 8;      // tile extent (voxels)
constexpr int kMaxLevels = 4;                   // 3 (16/32/64 channels) or 4 (16/32/64/128)
constexpr int kInCh = 16;                       // network input channels (4 used, rest zero)

// One 3x3x3 convolution launch over the active tiles of one level.
struct ConvArgs {
  int nx, ny, nz;              // level grid
  int ntx, nty, ntz;           // tiles per axis
  const int* tiles;            // active tile ids (t = (tz * nty + ty) * ntx + tx)
  const int* nTiles;           // device count of active tiles
  const uint8_t* active;       // activity of every tile of this level
  // input channels [0, c0) from src0 (upsampled x2 from the coarser level when
  // up0), [c0, c0 + c1) from src1; c0, c1 multiples of 8, c0 + c1 of 16
  const bf16* src0; int c0; int up0;
  const bf16* src1; int c1;
  const bf16* w;               // [cin/16][27][2][cout][8] (B operand, K-major chunks)
  const float* bias;           // [cout] (mode 0)
  int mode;                    // 0: bias + ReLU; 1: raw (backward data)
  const bf16* mask;            // mode 1: multiply by (mask > 0), same layout as the output; may be null
  bf16* out0; int split;       // channels [0, split) -> out0 (stride split)
  bf16* out1;                  // channels [split, cout) -> out1 (stride cout - split)
  int* err;
};

// tcgen05 implicit-GEMM convolution (ws_unet_conv.cu); cout in {16, 32, 48, 64, 96, 128, 192}
cudaError_t launch_conv3(const ConvArgs& a, int cout, int maxTiles, cudaStream_t s);
size_t conv3_smem_bytes(int cout);
int conv3_zt(int cout);
cudaError_t conv3_init();
// tcgen05 weight and bias gradients of one convolution (ws_unet_conv.cu);
// src describes the convolution's input as for launch_conv3, cout <= 128
// (in passes of 64 output channels)
cudaError_t launch_dw_tc(const ConvArgs& src, const bf16* dz, int cout, float* dw, float* db, int maxItems,
                         cudaStream_t s);

}  // namespace unet

namespace unet {

struct LayerSpec { const char* name; int level, c0, c1, cout; };
constexpr int kMaxLayers = 4 * (kMaxLevels - 1) + 2;
// The layers of an L-level network in forward order: per level l < L - 1 the
// encoder pair e<l>a, e<l>b (16 << l channels), the bottleneck pair ba, bb
// at level L - 1, then per level l = L - 2 .. 0 the decoder pair d<l>a
// (the upsampled level l + 1 output and the skip s<l> concatenated), d<l>b.
// Returns the layer count (4 L - 2).
int unet_layers(int levels, LayerSpec* out);

// grid and tiling of one level
struct Level {
  int nx, ny, nz, ntx, nty, ntz, ntiles;
  long long nvox;
};

// The network, its parameters (FP32 master + Adam state + packed BF16
// operands), per-level activations and gradients, and the store of
// (input, converged pressure) training pairs. Pairs are kept over the
// active level-0 tiles only: per pair its tile list and, per tile, the 1024
// voxels' normalised residual, cell type and target.
class Net {
 public:
  cudaError_t create(const Dims& d, int levels);
  void destroy();
  cudaError_t init_weights(uint32_t seed, cudaStream_t s);
  cudaError_t set_weights(const float* host, cudaStream_t s);
  cudaError_t set_gain(double g, cudaStream_t s);
  cudaError_t predict(float* q, const float* rhs, const uint8_t* diag8, const uint8_t* type, cudaStream_t s);
  cudaError_t reserve_pairs(int capacity, const uint8_t* type, cudaStream_t s);
  cudaError_t collect_pre(const float* q, const float* rhs, const uint8_t* diag8, const uint8_t* type, cudaStream_t s);
  cudaError_t collect_post(const float* q, cudaStream_t s);
  cudaError_t train(int steps, int batch, double lr, uint32_t seed, double* meanLoss, cudaStream_t s);
  cudaError_t accumulate(int samples, uint32_t seed, cudaStream_t s);
  cudaError_t apply(double lr, int total, cudaStream_t s);
  cudaError_t loss_sum(double* out, cudaStream_t s);
  cudaError_t forward_pair(int p, float* outHost, cudaStream_t s);
  cudaError_t grad_pair(int p, float* gradHost, double* loss, cudaStream_t s);
  // dense copies of a stored pair (zero / air outside its tiles), and a pair from dense arrays
  cudaError_t get_pair(int p, float* r0nHost, uint8_t* typeHost, float* targetHost, cudaStream_t s);
  cudaError_t put_pair(const float* r0nHost, const uint8_t* typeHost, const float* targetHost, cudaStream_t s);
  long long layer_weights(int l) const;
  int stored() const { return pairsStored < pairCap ? pairsStored : pairCap; }

  Dims dims{};
  int levels = 3, nLayers = 0;
  LayerSpec layers[kMaxLayers]{};
  long long nparams = 0, woff[kMaxLayers]{}, boff[kMaxLayers]{}, headOff = 0;
  float *params = nullptr, *grads = nullptr, *adm = nullptr, *adv = nullptr;
  int adamStep = 0;
  long long trainSteps = 0;
  double gain = 0, lastLoss = 0;
  // pair store: per slot tileCap tiles of 1024 voxels (r0 / sigma, type,
  // target), the tile ids, (tile count, fluid count), (sigma, sum target^2)
  float *pr0n = nullptr, *ptarget = nullptr;
  uint8_t* ptype = nullptr;
  int *ptiles = nullptr, *pmeta = nullptr;
  double* pscal = nullptr;
  int pairCap = 0, pairsStored = 0, tileCap = 0;
  long long pairsDropped = 0;       // pairs with more active tiles than a slot holds (not stored)
  int pendingSlot = -1;             // slot filled by collect_pre, awaiting its target
  int* err = nullptr;

 private:
  cudaError_t pack(cudaStream_t s);
  cudaError_t activity(const uint8_t* type, cudaStream_t s);
  cudaError_t lists(cudaStream_t s);
  cudaError_t residual(const float* q, const float* rhs, const uint8_t* diag8, const uint8_t* type, float* dst,
                       double* sig, cudaStream_t s, bool scale = true);
  cudaError_t unpack(int p, cudaStream_t s);
  cudaError_t conv(int l, const bf16* src0, const bf16* src1, bf16* out, cudaStream_t s);
  cudaError_t conv_bwd(int l, const bf16* dz, const bf16* mask, bf16* out0, bf16* out1, cudaStream_t s);
  cudaError_t dw(int l, const bf16* src0, const bf16* src1, const bf16* dz, cudaStream_t s);
  cudaError_t pool(int fineLevel, const bf16* fine, bf16* coarse, int ch, cudaStream_t s);
  cudaError_t forward(cudaStream_t s);
  cudaError_t backward(cudaStream_t s);
  cudaError_t sample_grad(int p, cudaStream_t s);
  cudaError_t set_gain_from_pairs(cudaStream_t s);
  int enc_a(int l) const { return 2 * l; }
  int enc_b(int l) const { return 2 * l + 1; }
  int bot_a() const { return 2 * (levels - 1); }
  int bot_b() const { return 2 * (levels - 1) + 1; }
  int dec_a(int l) const { return 2 * (levels - 1) + 2 + 2 * (levels - 2 - l); }
  int dec_b(int l) const { return dec_a(l) + 1; }
  int ch(int l) const { return 16 << l; }

  Level lv[kMaxLevels]{};
  uint8_t* act[kMaxLevels]{};
  int* tiles[kMaxLevels]{};
  int* counts = nullptr;          // tile counts of the levels, then (at kMaxLevels) the fluid-cell count
  // activations (level l, 16 << l channels unless noted): x (level 0, 16
  // input channels), ea/s (encoder outputs, s the skip), p (level l >= 1:
  // the pooled level l - 1 skip), bA/bB (bottleneck), da/db (decoder; h = db[0])
  bf16 *x = nullptr, *ea[kMaxLevels]{}, *sk[kMaxLevels]{}, *pl[kMaxLevels]{}, *bA = nullptr, *bB = nullptr;
  bf16 *da[kMaxLevels]{}, *db[kMaxLevels]{};
  // gradients: gdb (gh = gdb[0]), gda, gup (level l, 16 << (l + 1) channels:
  // the upsampled input of d<l>a), gsa (its skip part), gbA/gbB, gp, gs, gea
  bf16 *gdb[kMaxLevels]{}, *gda[kMaxLevels]{}, *gup[kMaxLevels]{}, *gsa[kMaxLevels]{}, *gbA = nullptr, *gbB = nullptr;
  bf16 *gp[kMaxLevels]{}, *gs[kMaxLevels]{}, *gea[kMaxLevels]{};
  bf16 *fw[kMaxLayers]{}, *bw[kMaxLayers]{};
  double* partials = nullptr;
  int nPartials = 0;
  double* scal = nullptr;         // sigma, gain, loss sum
  float *r0n = nullptr, *qprev = nullptr, *tscaled = nullptr, *outbuf = nullptr, *tbuf = nullptr;
  uint8_t* typebuf = nullptr;     // cell types of an unpacked pair
};

}  // namespace unet
