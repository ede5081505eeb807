// ws_unet.cuh — the learned warm start of the pressure solve: a small 3D
// U-Net (3 levels, 16/32/64 channels, 3x3x3 convolutions, BF16 weights and
// activations, FP32 accumulation in tensor memory) that predicts the change
// of the pressure over one solve from the initial residual. The reference
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
constexpr int kLevels = 3;
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

// tcgen05 implicit-GEMM convolution (ws_unet_conv.cu); cout in {16, 32, 48, 64, 96}
cudaError_t launch_conv3(const ConvArgs& a, int cout, int maxTiles, cudaStream_t s);
size_t conv3_smem_bytes(int cout);
int conv3_zt(int cout);
cudaError_t conv3_init();
// tcgen05 weight and bias gradients of one convolution (ws_unet_conv.cu);
// src describes the convolution's input as for launch_conv3, cout <= 128
cudaError_t launch_dw_tc(const ConvArgs& src, const bf16* dz, int cout, float* dw, float* db, int maxItems,
                         cudaStream_t s);

}  // namespace unet

namespace unet {

struct LayerSpec { const char* name; int level, c0, c1, cout; };
constexpr int kNumLayers = 10;
extern const LayerSpec kLayers[kNumLayers];

// grid and tiling of one level
struct Level {
  int nx, ny, nz, ntx, nty, ntz, ntiles;
  long long nvox;
};

// The network, its parameters (FP32 master + Adam state + packed BF16
// operands), per-level activations and gradients, and the store of
// (input, converged pressure) training pairs.
class Net {
 public:
  cudaError_t create(const Dims& d);
  void destroy();
  cudaError_t init_weights(uint32_t seed, cudaStream_t s);
  cudaError_t set_weights(const float* host, cudaStream_t s);
  cudaError_t set_gain(double g, cudaStream_t s);
  cudaError_t predict(float* q, const float* rhs, const uint8_t* diag8, const uint8_t* type, cudaStream_t s);
  cudaError_t reserve_pairs(int capacity);
  cudaError_t collect_pre(const float* q, const float* rhs, const uint8_t* diag8, const uint8_t* type, cudaStream_t s);
  cudaError_t collect_post(const float* q, cudaStream_t s);
  cudaError_t train(int steps, int batch, double lr, uint32_t seed, double* meanLoss, cudaStream_t s);
  cudaError_t accumulate(int samples, uint32_t seed, cudaStream_t s);
  cudaError_t apply(double lr, int total, cudaStream_t s);
  cudaError_t loss_sum(double* out, cudaStream_t s);
  cudaError_t forward_pair(int p, float* outHost, cudaStream_t s);
  cudaError_t grad_pair(int p, float* gradHost, double* loss, cudaStream_t s);
  static long long layer_weights(int l);

  Dims dims{};
  long long nparams = 0, woff[kNumLayers]{}, boff[kNumLayers]{}, headOff = 0;
  float *params = nullptr, *grads = nullptr, *adm = nullptr, *adv = nullptr;
  int adamStep = 0;
  long long trainSteps = 0;
  double gain = 0, lastLoss = 0;
  // pair store: r0 / sigma, cell types, target, and (sigma, sum target^2) per pair
  float *pr0n = nullptr, *ptarget = nullptr;
  uint8_t* ptype = nullptr;
  double* pscal = nullptr;
  int pairCap = 0, pairsStored = 0;
  int* err = nullptr;

 private:
  cudaError_t pack(cudaStream_t s);
  cudaError_t activity(const uint8_t* type, cudaStream_t s);
  cudaError_t residual(const float* q, const float* rhs, const uint8_t* diag8, const uint8_t* type, float* dst,
                       double* sig, cudaStream_t s, bool scale = true);
  cudaError_t prepare(const float* r0nIn, const uint8_t* type, cudaStream_t s);
  cudaError_t conv(int l, const bf16* src0, const bf16* src1, bf16* out, cudaStream_t s);
  cudaError_t conv_bwd(int l, const bf16* dz, const bf16* mask, bf16* out0, bf16* out1, cudaStream_t s);
  cudaError_t dw(int l, const bf16* src0, const bf16* src1, const bf16* dz, cudaStream_t s);
  cudaError_t pool(int fineLevel, const bf16* fine, bf16* coarse, int ch, cudaStream_t s);
  cudaError_t forward(cudaStream_t s);
  cudaError_t backward(cudaStream_t s);
  cudaError_t sample_grad(int p, cudaStream_t s);
  cudaError_t set_gain_from_pairs(cudaStream_t s);

  Level lv[kLevels]{};
  uint8_t* act[kLevels]{};
  int* tiles[kLevels]{};
  int* counts = nullptr;          // tile counts of the levels, then the fluid-cell count
  bf16 *x = nullptr, *e0a = nullptr, *s0 = nullptr, *d0a = nullptr, *h = nullptr;
  bf16 *gh = nullptr, *gd0a = nullptr, *gs0a = nullptr, *gs0 = nullptr, *ge0a = nullptr, *gup1 = nullptr;
  bf16 *p1 = nullptr, *gp1 = nullptr, *e1a = nullptr, *s1 = nullptr, *d1a = nullptr, *d1b = nullptr;
  bf16 *gd1b = nullptr, *gd1a = nullptr, *gs1a = nullptr, *gs1 = nullptr, *ge1a = nullptr, *gup2 = nullptr;
  bf16 *p2 = nullptr, *gp2 = nullptr, *ba = nullptr, *bb = nullptr, *gbb = nullptr, *gba = nullptr;
  bf16 *fw[kNumLayers]{}, *bw[kNumLayers]{};
  double* partials = nullptr;
  int nPartials = 0;
  double* scal = nullptr;         // sigma, gain, loss sum
  float *r0n = nullptr, *qprev = nullptr, *tscaled = nullptr, *outbuf = nullptr;
};

}  // namespace unet
