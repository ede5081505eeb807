// ws_noalloc.cu — ws_residual_noalloc: the FP64 divergence residual of the
// pressure system without any device allocation.
//
// Who needs it: callers that own every device buffer themselves and cannot
// let a library call cudaMalloc. Examples are a host that sizes all GPU memory
// up front through its own allocator (the reference's `alloc(name, ctor,
// len)` hook is that seam), and a frame loop where cudaMalloc/cudaFree would
// synchronise the device and stall the frame. Creating a ws_handle
// allocates, so this entry point takes the caller's own q, rhs and cellType
// buffers and writes the result to the caller's own device double.
//
// Scratch: one block partial per 256 cells lives in the file-scope array
// g_noalloc_partials below (128 KB, held by every GPU that loads the
// library until the process exits). Grids above WS_NOALLOC_MAX_CELLS cells
// are rejected with WS_ERR_RANGE before anything is launched. Every call
// writes every partial it reads, so nothing has to start at zero. All calls
// on one device share the array: calls whose kernels overlap on the GPU (two
// streams, two host threads) race and must be serialised by the caller.
//
// Set-up: the first call on each device, with that device current, looks the
// array's device address up with cudaGetSymbolAddress (host code must not
// pass the symbol itself to a kernel). Make that first call before any
// stream capture.
#include "ws_kernels.cuh"
#include <atomic>

#define WS_NOALLOC_BLOCK 256
#define WS_NOALLOC_MAX_BLOCKS 8192
#define WS_NOALLOC_MAX_CELLS ((long long)WS_NOALLOC_BLOCK * WS_NOALLOC_MAX_BLOCKS)   // 128^3

static __device__ __align__(256) double2 g_noalloc_partials[WS_NOALLOC_MAX_BLOCKS];

// r = rhs + sum of fluid-neighbour q - diag q over interior fluid cells,
// diag = number of non-solid neighbours (js/solver.js:1342-1365)
__global__ void __launch_bounds__(WS_NOALLOC_BLOCK) k_noalloc_partial(int nx, int ny, int nz,
    const float* __restrict__ q, const float* __restrict__ rhs, const uint8_t* __restrict__ type,
    double2* __restrict__ partials) {
  __shared__ double srr[32], sbb[32];
  unsigned c = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned N = (unsigned)nx * ny * nz;
  double rr = 0, bb = 0;
  if (c < N && type[c] == WS_FLUID) {
    unsigned t = c / nx, i = c - t * nx, k = t / ny, j = t - k * ny;
    if (i > 0 && j > 0 && k > 0 && (int)i < nx - 1 && (int)j < ny - 1 && (int)k < nz - 1) {
      long long nxy = (long long)nx * ny;
      long long nb[6] = { (long long)c - 1, (long long)c + 1, (long long)c - nx, (long long)c + nx,
                          (long long)c - nxy, (long long)c + nxy };
      double sum = 0; int diag = 0;
      for (int d = 0; d < 6; d++) {
        int tn = type[nb[d]];
        if (tn != WS_SOLID) diag++;
        if (tn == WS_FLUID) sum += (double)q[nb[d]];
      }
      double b = rhs[c];
      double r = b + sum - (double)diag * (double)q[c];
      rr = r * r; bb = b * b;
    }
  }
  rr = warp_sum(rr); bb = warp_sum(bb);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { srr[wid] = rr; sbb[wid] = bb; }
  __syncthreads();
  if (wid == 0) {
    rr = lane < (int)(blockDim.x >> 5) ? srr[lane] : 0; bb = lane < (int)(blockDim.x >> 5) ? sbb[lane] : 0;
    rr = warp_sum(rr); bb = warp_sum(bb);
    if (lane == 0) partials[blockIdx.x] = make_double2(rr, bb);   // every slot read below is written here
  }
}
// fixed-order sum of the partials -> ||r|| / ||b|| (||r|| when b = 0)
__global__ void k_noalloc_final(const double2* __restrict__ partials, int n, double* __restrict__ out) {
  __shared__ double srr[32], sbb[32];
  double rr = 0, bb = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) { rr += partials[i].x; bb += partials[i].y; }
  rr = warp_sum(rr); bb = warp_sum(bb);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { srr[wid] = rr; sbb[wid] = bb; }
  __syncthreads();
  if (wid == 0) {
    rr = lane < (int)(blockDim.x >> 5) ? srr[lane] : 0; bb = lane < (int)(blockDim.x >> 5) ? sbb[lane] : 0;
    rr = warp_sum(rr); bb = warp_sum(bb);
    if (lane == 0) *out = bb > 0 ? sqrt(rr) / sqrt(bb) : sqrt(rr);
  }
}

// device address of g_noalloc_partials, looked up once per device
static std::atomic<double2*> s_scratch[256];

extern "C" ws_status ws_residual_noalloc(int32_t nx, int32_t ny, int32_t nz, const float* q, const float* rhs,
                                         const uint8_t* cellType, double* relres, void* stream) {
  if (nx < 3 || ny < 3 || nz < 3 || !q || !rhs || !cellType || !relres) return WS_ERR_INVALID;
  long long cells = (long long)nx * ny * nz;
  if (cells > WS_NOALLOC_MAX_CELLS) return WS_ERR_RANGE;        // beyond the fixed scratch
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) return WS_ERR_CUDA;
  double2* scratch = s_scratch[dev].load(std::memory_order_acquire);
  if (!scratch) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_partials) != cudaSuccess || !p) return WS_ERR_CUDA;
    scratch = (double2*)p;
    s_scratch[dev].store(scratch, std::memory_order_release);
  }
  cudaStream_t s = (cudaStream_t)stream;
  int nb = (int)((cells + WS_NOALLOC_BLOCK - 1) / WS_NOALLOC_BLOCK);
  k_noalloc_partial<<<nb, WS_NOALLOC_BLOCK, 0, s>>>(nx, ny, nz, q, rhs, cellType, scratch);
  k_noalloc_final<<<1, 1024, 0, s>>>(scratch, nb, relres);
  return cudaGetLastError() == cudaSuccess ? WS_OK : WS_ERR_CUDA;
}
