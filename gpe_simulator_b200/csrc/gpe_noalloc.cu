// gpe_noalloc.cu -- renormalisation that allocates no device memory.
//
// gpe_normalise() needs a plan, and creating a plan calls cudaMalloc for its
// tables and for the scratch of the norm reduction (per-block partial sums, a
// completion ticket and the resulting scale).  Some callers cannot allocate:
// host frameworks that own the GPU memory pool (a caching allocator or a
// preallocated arena that has already reserved the free HBM, where a stray
// cudaMalloc fails or fragments the pool), and plugin hosts that forbid
// allocation inside their per-step callbacks.  gpe_normalise_noalloc() serves
// them: the same compensated FP64 norm reduction and in-place division, with
// the scratch in a file-scope __device__ array instead of plan buffers.
//
// Limits and sharing:
//  * grids up to 1024^3 points (n <= 1024); the reduction runs on at most
//    GPE_NOALLOC_BLOCKS blocks, so the scratch is a fixed 16 KiB per device;
//  * every GPU that loads the library holds the array until the process exits;
//  * all calls on a device share the one array, which keeps the last call's
//    contents: the completion ticket and status word are cleared at the start
//    of every call, and calls whose work overlaps on the GPU (different streams,
//    no ordering between them) race on it -- serialise them;
//  * the first call on each device looks up the array's device address with
//    cudaGetSymbolAddress (module set-up); make that first call before any
//    stream capture.
#include "../../include/gpe_ssf.h"
#include "gpe_kernels.cuh"

#include <cmath>
#include <cstdio>
#include <string>

using namespace gpe;

namespace gpe {
void set_last_error(const std::string& msg);  // gpe_last_error() reports it (gpe_ssf.cu)
}

namespace {

constexpr int GPE_NOALLOC_BLOCKS = 1184;     // 8 blocks per SM on 148 SMs
constexpr int GPE_NOALLOC_THREADS = 256;

// [0, 8*BLOCKS)        per-block partial sums (double)
// [8*BLOCKS, +32)      sqrt(N), 1/sqrt(N), N, spare (double x4)
// [8*BLOCKS + 32, +4)  completion ticket (unsigned)
// [8*BLOCKS + 36, +4)  status word (int)
constexpr size_t SCRATCH_BYTES = 16384;
static_assert(8 * GPE_NOALLOC_BLOCKS + 40 <= SCRATCH_BYTES, "scratch too small");

__device__ __align__(256) unsigned char g_noalloc_scratch[SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
void* g_scratch_ptr[MAX_DEVICES] = {nullptr};

int fail_na(int code, const std::string& msg) {
  gpe::set_last_error(msg);
  return code;
}

// Device address of the scratch array on the current device (set-up on first use).
int scratch_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail_na(GPE_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= MAX_DEVICES) return fail_na(GPE_ERR_UNSUPPORTED, "device index out of range");
  if (!g_scratch_ptr[dev]) {
    void* ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess)
      return fail_na(GPE_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratch_ptr[dev] = ptr;
  }
  *out = g_scratch_ptr[dev];
  return GPE_OK;
}

// Grid-stride variant of the sweeps' norm reduction: per-thread compensated
// sums of |psi|^2, a fixed-order block merge, and the last block to finish sums
// the block partials in index order (deterministic) and stores sqrt(N).
template <typename R>
__global__ void __launch_bounds__(GPE_NOALLOC_THREADS)
k_norm_noalloc(const typename Cx<R>::T* __restrict__ psi, long long m, double dx3, unsigned char* scratch) {
  __shared__ Acc sh[32];
  __shared__ bool last;
  double* partial = (double*)scratch;
  double* scale = partial + GPE_NOALLOC_BLOCKS;
  unsigned* ticket = (unsigned*)(scale + 4);
  int* status = (int*)(ticket + 1);
  Acc a[1];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m;
       i += (long long)gridDim.x * blockDim.x) {
    const typename Cx<R>::T v = psi[i];
    a[0].add((double)v.x * v.x + (double)v.y * v.y);
  }
  block_merge<1>(a, sh);
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = a[0].value();
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  Acc t[1];
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) t[0].add(__ldcg(partial + b));
  block_merge<1>(t, sh);
  if (threadIdx.x == 0) {
    const double N = t[0].value() * dx3;
    if (!(N > 0.0) || !isfinite(N)) atomicOr(status, ST_NONFINITE);
    scale[0] = sqrt(N);
    scale[1] = 1.0 / scale[0];
    scale[2] = N;
    *ticket = 0u;
  }
}

// psi /= sqrt(N) (reference gpe/helper.py:93), reading sqrt(N) from the scratch.
template <typename R>
__global__ void __launch_bounds__(GPE_NOALLOC_THREADS)
k_scale_noalloc(typename Cx<R>::T* __restrict__ psi, long long m, const unsigned char* scratch) {
  const double* scale = (const double*)scratch + GPE_NOALLOC_BLOCKS;
  const double s = __ldcg(scale);
  const R inv = (R)__ldcg(scale + 1);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m;
       i += (long long)gridDim.x * blockDim.x) {
    typename Cx<R>::T v = psi[i];
    if (sizeof(R) == 8) { v.x = (R)((double)v.x / s); v.y = (R)((double)v.y / s); }
    else { v.x *= inv; v.y *= inv; }
    psi[i] = v;
  }
}

}  // namespace

extern "C" int gpe_normalise_noalloc(void* psi, int n, int dtype, double dx, double* norm, void* stream) {
  if (!psi) return fail_na(GPE_ERR_ARG, "null psi");
  if (n < 1 || n > 1024)
    return fail_na(GPE_ERR_UNSUPPORTED, "gpe_normalise_noalloc: n must be in [1, 1024] (at most 2^30 points)");
  if (dtype != GPE_C64 && dtype != GPE_C128) return fail_na(GPE_ERR_ARG, "dtype must be GPE_C64 or GPE_C128");
  if (!(dx > 0.0) || !std::isfinite(dx)) return fail_na(GPE_ERR_ARG, "dx must be positive and finite");
  void* scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc != GPE_OK) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  unsigned char* base = (unsigned char*)scratch;
  // the ticket and the status word must start at zero
  cudaError_t e = cudaMemsetAsync(base + 8 * GPE_NOALLOC_BLOCKS + 32, 0, 8, st);
  if (e != cudaSuccess) return fail_na(GPE_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
  const long long m = (long long)n * n * n;
  long long want = (m + GPE_NOALLOC_THREADS - 1) / GPE_NOALLOC_THREADS;
  const int blocks = (int)(want < GPE_NOALLOC_BLOCKS ? want : GPE_NOALLOC_BLOCKS);
  const double dx3 = dx * dx * dx;
  if (dtype == GPE_C64) {
    k_norm_noalloc<float><<<blocks, GPE_NOALLOC_THREADS, 0, st>>>((const float2*)psi, m, dx3, base);
    k_scale_noalloc<float><<<blocks, GPE_NOALLOC_THREADS, 0, st>>>((float2*)psi, m, base);
  } else {
    k_norm_noalloc<double><<<blocks, GPE_NOALLOC_THREADS, 0, st>>>((const double2*)psi, m, dx3, base);
    k_scale_noalloc<double><<<blocks, GPE_NOALLOC_THREADS, 0, st>>>((double2*)psi, m, base);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail_na(GPE_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  if (norm) {
    e = cudaMemcpyAsync(norm, base + 8 * GPE_NOALLOC_BLOCKS + 16, sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail_na(GPE_ERR_CUDA, std::string("read back: ") + cudaGetErrorString(e));
  }
  return GPE_OK;
}
