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
// Set-up: host code must not hand the array's name to a kernel (on the host it
// names a stand-in, not device memory). Every call therefore looks up the
// array's device address with cudaGetSymbolAddress on the current device and
// checks the result. The lookup allocates nothing; repeating it on every call
// keeps the address right when the caller's context is re-created (after
// cudaDeviceReset the library's device code is loaded again, possibly at
// another address). The first call on a device also loads the library's
// device code there, so it should come before any stream capture. The
// entry point uses the runtime's current (primary) context of the current
// device.
//
// Errors: each of the two launches is checked through its own return code
// (cudaLaunchKernel). The calling thread's pending CUDA error state is left
// as it was: an earlier, unrelated error is neither cleared nor reported as
// this call's.
#include "ws_kernels.cuh"

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

extern "C" ws_status ws_residual_noalloc(int32_t nx, int32_t ny, int32_t nz, const float* q, const float* rhs,
                                         const uint8_t* cellType, double* relres, void* stream) {
  if (nx < 3 || ny < 3 || nz < 3 || !q || !rhs || !cellType || !relres) return WS_ERR_INVALID;
  long long cells = (long long)nx * ny * nz;
  if (cells > WS_NOALLOC_MAX_CELLS) return WS_ERR_RANGE;        // beyond the fixed scratch
  void* sp = nullptr;
  if (cudaGetSymbolAddress(&sp, g_noalloc_partials) != cudaSuccess || !sp) return WS_ERR_CUDA;
  double2* scratch = (double2*)sp;
  cudaStream_t s = (cudaStream_t)stream;
  int nb = (int)((cells + WS_NOALLOC_BLOCK - 1) / WS_NOALLOC_BLOCK);
  void* a1[] = { &nx, &ny, &nz, (void*)&q, (void*)&rhs, (void*)&cellType, &scratch };
  if (cudaLaunchKernel((const void*)k_noalloc_partial, dim3(nb), dim3(WS_NOALLOC_BLOCK), a1, 0, s) != cudaSuccess)
    return WS_ERR_CUDA;
  void* a2[] = { &scratch, &nb, &relres };
  if (cudaLaunchKernel((const void*)k_noalloc_final, dim3(1), dim3(1024), a2, 0, s) != cudaSuccess)
    return WS_ERR_CUDA;
  return WS_OK;
}
