// Residual norm that allocates nothing.
//
// Some callers cannot call cudaMalloc at the point where they need the norm: a host solver
// whose device memory is owned by another allocator (a caching pool or a fixed arena that must
// see every byte), or a time-critical pseudo-time loop that cannot afford the implicit
// device-wide synchronisation of cudaMalloc/cudaFree. rds_residual_norm_noalloc serves them:
// it reads the caller's residual and time-step arrays, writes the caller's output, and keeps
// its per-block partial sums in a fixed array in this library's device memory
// (g_norm_partials below) instead of allocating scratch.
//
// The array's address is taken once per device with cudaGetSymbolAddress (host code cannot use
// the symbol itself: in host code it names a host-side stand-in, not device memory). That
// set-up happens in the first call on each device, so the first call on a device must come
// before any stream capture. The cached address is not looked up again: a cudaDeviceReset
// (which unloads the module) makes it stale, so a process that resets a device does not call
// this entry point on that device afterwards. All calls share the array: calls that overlap on
// the GPU (two streams, two host threads) race on it. Every partial that a call reads was
// written by the same call, so nothing has to start at zero.

#include <mutex>

#include "rds_internal.h"

namespace
{

constexpr int kNT = rds::kGBlock; // 256 nodes per block, as rds_residual_norm

// Per-block partial sums, [block][neq]: RDS_NOALLOC_MAX_NODES / 256 blocks x 5 equations
// (32768 x 5 doubles = 1.25 MiB of device memory held by every GPU that loads the library).
static __device__ __align__(256) double g_norm_partials[(RDS_NOALLOC_MAX_NODES / kNT) * 5];

constexpr int kMaxDevices = 64;
double *g_partials_ptr[kMaxDevices] = {};
std::mutex g_setup_mutex;

__device__ __forceinline__ double block_sum_na(double v, double *smem)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0)
    smem[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kNT / 32; ++w)
      s += smem[w];
  return s;
}

// Same block decomposition and summation order as rds_residual_norm, so both give the same
// bits for the same inputs.
__global__ void __launch_bounds__(kNT)
    norm_partials_na(int nnodes, int neq, const double *res, const double *dt, double *part)
{
  __shared__ double smem[kNT / 32];
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  for (int e = 0; e < neq; ++e)
  {
    double sq = 0.0;
    if (v < nnodes)
    {
      const double r = __dmul_rn(res[(size_t)e * nnodes + v], dt[v]);
      sq             = __dmul_rn(r, r);
    }
    const double s = block_sum_na(sq, smem);
    if (threadIdx.x == 0)
      part[(size_t)blockIdx.x * neq + e] = s;
  }
}

__global__ void __launch_bounds__(kNT)
    norm_final_na(const double *part, int nblocks, int neq, int nnodes, double *norm)
{
  __shared__ double smem[kNT / 32];
  for (int e = 0; e < neq; ++e)
  {
    double s = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
      s += part[(size_t)b * neq + e];
    s = block_sum_na(s, smem);
    if (threadIdx.x == 0)
      norm[e] = sqrt(s / nnodes);
  }
}

// Device address of g_norm_partials for the current device (set up on first use).
rds_status partials_for_current_device(double **out)
{
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return RDS_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_partials_ptr[dev])
  {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_norm_partials) != cudaSuccess || !p)
      return RDS_ERR_CUDA;
    g_partials_ptr[dev] = static_cast<double *>(p);
  }
  *out = g_partials_ptr[dev];
  return RDS_OK;
}

} // namespace

extern "C" RDS_API rds_status rds_residual_norm_noalloc(const double *res, const double *dt,
                                                        int nnodes, int neq, double *norm,
                                                        void *stream)
{
  if (!res || !dt || !norm || nnodes <= 0 || neq < 1 || neq > 5)
    return RDS_ERR_INVALID;
  if (nnodes > RDS_NOALLOC_MAX_NODES)
    return RDS_ERR_TOO_LARGE;
  double *part      = nullptr;
  const rds_status st = partials_for_current_device(&part);
  if (st != RDS_OK)
    return st;
  cudaStream_t s    = static_cast<cudaStream_t>(stream);
  const int nblocks = (nnodes + kNT - 1) / kNT;
  norm_partials_na<<<nblocks, kNT, 0, s>>>(nnodes, neq, res, dt, part);
  norm_final_na<<<1, kNT, 0, s>>>(part, nblocks, neq, nnodes, norm);
  return cudaGetLastError() == cudaSuccess ? RDS_OK : RDS_ERR_CUDA;
}
