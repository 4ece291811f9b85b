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
//  * set-up happens on the first call in each CUDA context (normally one per
//    device): it looks up the array's device address with cudaGetSymbolAddress
//    and loads this file's four kernels, so that no later call loads code (with
//    CUDA's lazy module loading a first launch would otherwise load it, taking
//    device memory); make that first call before any stream capture.  The
//    address is cached per context id, so a context torn down and created again
//    (cudaDeviceReset) gets a fresh look-up instead of a stale address;
//  * every call synchronises `stream`: it reads the status word back and
//    returns GPE_ERR_NONFINITE, with psi left unchanged, when N is zero, NaN or
//    infinite.
#include "../../include/gpe_ssf.h"
#include "gpe_kernels.cuh"

#include <cuda.h>

#include <cmath>
#include <cstdio>
#include <mutex>
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

int fail_na(int code, const std::string& msg) {
  gpe::set_last_error(msg);
  return code;
}

// Context id of the calling thread's current context (cuCtxGetCurrent +
// cuCtxGetId from the driver, reached through the runtime's entry-point query,
// so the library needs no link-time dependency on libcuda).
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

int current_context_id(unsigned long long* id) {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  if (!get_current || !get_id) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return fail_na(GPE_ERR_CUDA, "cuCtxGetCurrent is not available from the driver");
    get_current = (CtxGetCurrentFn)f;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return fail_na(GPE_ERR_CUDA, "cuCtxGetId is not available from the driver");
    get_id = (CtxGetIdFn)f;
  }
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return fail_na(GPE_ERR_CUDA, "no current CUDA context");
  if (get_id(ctx, id) != CUDA_SUCCESS) return fail_na(GPE_ERR_CUDA, "cuCtxGetId failed");
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

// psi /= sqrt(N) (reference gpe/helper.py:93), reading sqrt(N) from the scratch;
// nothing is written when the norm kernel flagged N as zero or non-finite.
template <typename R>
__global__ void __launch_bounds__(GPE_NOALLOC_THREADS)
k_scale_noalloc(typename Cx<R>::T* __restrict__ psi, long long m, const unsigned char* scratch) {
  const double* scale = (const double*)scratch + GPE_NOALLOC_BLOCKS;
  const int* status = (const int*)((const unsigned*)(scale + 4) + 1);
  if (__ldcg(status) & ST_NONFINITE) return;   // zero or non-finite N: psi left as it is
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

// Scratch address per CUDA context (a context id is never reused in a process).
constexpr int MAX_CONTEXTS = 64;
struct ScratchSlot { unsigned long long ctx; void* ptr; };
ScratchSlot g_slots[MAX_CONTEXTS] = {};
int g_nslots = 0;
std::mutex g_slots_mu;

// Device address of the scratch array in the current context; the first call
// in a context also loads this file's kernels (both precisions).
int scratch_address(void** out) {
  unsigned long long ctx = 0;
  int rc = current_context_id(&ctx);
  if (rc != GPE_OK) return rc;
  std::lock_guard<std::mutex> lock(g_slots_mu);
  for (int i = 0; i < g_nslots; ++i)
    if (g_slots[i].ctx == ctx) { *out = g_slots[i].ptr; return GPE_OK; }
  if (g_nslots == MAX_CONTEXTS) return fail_na(GPE_ERR_UNSUPPORTED, "too many CUDA contexts");
  void* ptr = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
  if (e != cudaSuccess) return fail_na(GPE_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  // load the kernels now (a lazily loaded module would load on first launch)
  cudaFuncAttributes fa;
  const void* fns[4] = {(const void*)k_norm_noalloc<float>, (const void*)k_scale_noalloc<float>,
                        (const void*)k_norm_noalloc<double>, (const void*)k_scale_noalloc<double>};
  for (const void* f : fns) {
    e = cudaFuncGetAttributes(&fa, f);
    if (e != cudaSuccess) return fail_na(GPE_ERR_CUDA, std::string("cudaFuncGetAttributes: ") + cudaGetErrorString(e));
  }
  g_slots[g_nslots++] = ScratchSlot{ctx, ptr};
  *out = ptr;
  return GPE_OK;
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
  // N, the spare slot, the ticket and the status word, read back in one copy
  struct { double N, spare; unsigned ticket; int status; } back;
  static_assert(sizeof(back) == 24, "read-back layout");
  e = cudaMemcpyAsync(&back, base + 8 * GPE_NOALLOC_BLOCKS + 16, sizeof(back), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail_na(GPE_ERR_CUDA, std::string("read back: ") + cudaGetErrorString(e));
  if (norm) *norm = back.N;
  if (back.status & ST_NONFINITE)
    return fail_na(GPE_ERR_NONFINITE, "gpe_normalise_noalloc: the norm is zero or not finite; psi is unchanged");
  return GPE_OK;
}
