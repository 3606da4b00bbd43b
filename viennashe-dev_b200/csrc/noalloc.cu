// noalloc.cu -- the one entry point of this library that allocates no device memory:
// r = b - A x and the squared norms ||r||^2, ||b||^2 of a caller-owned CSR system.
//
// Who needs it: callers whose device memory is owned by someone else -- a host application
// whose framework hands out every byte of HBM through its own arena or caching allocator, or a
// Gummel/Newton driver that must not call cudaMalloc inside its timed inner loop (cudaMalloc and
// cudaFree synchronise the device).  Such callers bring their own device buffers for the inputs
// and outputs; the only scratch this computation needs -- one pair of partial sums per tile of
// 2048 rows and a ticket counter for the last-tile reduction -- lives in a fixed file-scope
// __device__ array instead of a cudaMalloc'd buffer.
//
// The array is sized for kMaxTiles tiles (512 KiB of partial sums): at most 64 Mi rows.  Every
// GPU that loads this library holds it until the process exits.  All calls share it: two calls
// whose kernels overlap on the GPU (different streams, or different host threads on one
// device) race on it; calls on one stream are ordered and safe.  The partial sums are fully
// rewritten by every call; the ticket counter must start at zero, which the set-up clears
// once per device, and every call leaves it at zero again.
#include <cuda_runtime.h>
#include <cstdint>
#include <mutex>

#include "../../include/vshe_gpu.h"
#include "kernels.h"

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int64_t kTileRows = 2048;
constexpr int64_t kMaxTiles = 32768;
constexpr int kMaxDevices = 64;

struct NoAllocScratch {
  double partial[2 * kMaxTiles];  // (||r||^2, ||b||^2) of every tile
  unsigned int ticket;            // tiles finished in the current call
};

static __device__ __align__(256) NoAllocScratch g_scratch;

// Per-device address of g_scratch (host code cannot use the symbol itself as a pointer).
std::mutex g_mu;
NoAllocScratch *g_addr[kMaxDevices] = {nullptr};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// sums over the block, result valid in thread 0; fixed order (deterministic)
__device__ __forceinline__ void block_sum2(double &a, double &b) {
  __shared__ double sh[2][kWarps];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  a = warp_sum(a); b = warp_sum(b);
  if (lane == 0) { sh[0][w] = a; sh[1][w] = b; }
  __syncthreads();
  if (w == 0) {
    a = warp_sum(lane < kWarps ? sh[0][lane] : 0.0);
    b = warp_sum(lane < kWarps ? sh[1][lane] : 0.0);
  }
  __syncthreads();
}

// One block per tile of kTileRows rows, one warp per row in turn (lanes stride the row's entries,
// then a fixed-order warp sum).  The last tile to finish adds the tile partials in tile order.
__global__ void __launch_bounds__(kThreads) k_residual_noalloc(int64_t n, const int64_t *__restrict__ rp, const int32_t *__restrict__ ci,
                                                               const double *__restrict__ av, const double *__restrict__ x,
                                                               const double *__restrict__ b, double *__restrict__ r,
                                                               double *__restrict__ norms2, NoAllocScratch *sc) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t r0 = (int64_t)blockIdx.x * kTileRows;
  const int64_t r1 = r0 + kTileRows < n ? r0 + kTileRows : n;
  double rr = 0.0, bb = 0.0;
  for (int64_t i = r0 + w; i < r1; i += kWarps) {
    double s = 0.0;
    for (int64_t k = rp[i] + lane; k < rp[i + 1]; k += 32) s += av[k] * x[ci[k]];
    s = warp_sum(s);
    if (lane == 0) {
      const double bi = b[i];
      const double ri = bi - s;
      r[i] = ri;
      rr += ri * ri;
      bb += bi * bi;
    }
  }
  block_sum2(rr, bb);
  __shared__ int last;
  if (threadIdx.x == 0) {
    sc->partial[2 * blockIdx.x] = rr;
    sc->partial[2 * blockIdx.x + 1] = bb;
    __threadfence();
    last = (atomicAdd(&sc->ticket, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double ta = 0.0, tb = 0.0;
  for (int64_t t = threadIdx.x; t < gridDim.x; t += kThreads) {
    ta += ((volatile double *)sc->partial)[2 * t];
    tb += ((volatile double *)sc->partial)[2 * t + 1];
  }
  block_sum2(ta, tb);
  if (threadIdx.x == 0) {
    norms2[0] = ta;
    norms2[1] = tb;
    sc->ticket = 0;  // ready for the next call
  }
}

// Address of g_scratch on the current device; the first call on a device looks it up and
// clears the ticket counter.
int scratch_for_current_device(NoAllocScratch **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return VSHE_E_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return VSHE_E_UNSUPPORTED;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess) return VSHE_E_CUDA;
    NoAllocScratch *s = static_cast<NoAllocScratch *>(p);
    if (cudaMemset(&s->ticket, 0, sizeof(unsigned int)) != cudaSuccess) return VSHE_E_CUDA;
    if (cudaDeviceSynchronize() != cudaSuccess) return VSHE_E_CUDA;
    g_addr[dev] = s;
  }
  *out = g_addr[dev];
  return VSHE_OK;
}

}  // namespace

extern "C" int vshe_csr_residual_noalloc(int64_t n, int64_t nnz, const int64_t *d_row_ptr, const int32_t *d_col,
                                         const double *d_val, const double *d_x, const double *d_b, double *d_r,
                                         double *d_norms2, void *stream) {
  if (n <= 0 || nnz < 0 || !d_row_ptr || (nnz > 0 && (!d_col || !d_val)) || !d_x || !d_b || !d_r || !d_norms2)
    return VSHE_E_INVALID_ARGUMENT;
  if (n > kMaxTiles * kTileRows || n >= (int64_t(1) << 31)) return VSHE_E_CAPACITY;
  NoAllocScratch *sc = nullptr;
  int rc = scratch_for_current_device(&sc);
  if (rc) return rc;
  const int tiles = int((n + kTileRows - 1) / kTileRows);
  vk_count_launches(1);
  k_residual_noalloc<<<tiles, kThreads, 0, static_cast<cudaStream_t>(stream)>>>(n, d_row_ptr, d_col, d_val, d_x, d_b, d_r, d_norms2, sc);
  return cudaGetLastError() == cudaSuccess ? VSHE_OK : VSHE_E_CUDA;
}
