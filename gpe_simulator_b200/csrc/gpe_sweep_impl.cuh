// gpe_sweep_impl.cuh -- instantiation of the sweep kernels for one precision.
#pragma once
#include "gpe_sweep.h"

namespace gpe {

template <typename R, int AX, int EPT, bool GEN>
static cudaError_t launch_one(const Phys& ph, const Sweep& sw, int tiles, int threads, size_t smem,
                              cudaStream_t st) {
  static int attr_dev = -1;
  int dev = 0;
  cudaGetDevice(&dev);
  if (attr_dev != dev) {
    // opt-in limit minus the kernel's static shared memory
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, k_sweep<R, AX, EPT, GEN>);
    if (e != cudaSuccess) return e;
    int optin = 0;
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_sweep<R, AX, EPT, GEN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             optin - (int)fa.sharedSizeBytes);
    if (e != cudaSuccess) return e;
    attr_dev = dev;
  }
  k_sweep<R, AX, EPT, GEN><<<tiles, threads, smem, st>>>(ph, sw);
  return cudaGetLastError();
}

template <typename R>
cudaError_t launch_sweep(int ax, bool gen, const Phys& ph, const Sweep& sw, int tiles, int threads,
                         size_t smem, cudaStream_t st) {
  if (gen) {
    if (ax == AX_Z) return launch_one<R, AX_Z, 8, true>(ph, sw, tiles, threads, smem, st);
    if (ax == AX_Y) return launch_one<R, AX_Y, 8, true>(ph, sw, tiles, threads, smem, st);
    return launch_one<R, AX_X, 8, true>(ph, sw, tiles, threads, smem, st);
  }
  if (ax == AX_Z) return launch_one<R, AX_Z, 16, false>(ph, sw, tiles, threads, smem, st);
  if (ax == AX_Y) return launch_one<R, AX_Y, 16, false>(ph, sw, tiles, threads, smem, st);
  return launch_one<R, AX_X, 16, false>(ph, sw, tiles, threads, smem, st);
}

}  // namespace gpe

namespace gpe {

template <typename R, int AX, int EPT, bool GEN>
static cudaError_t launch_batch_one(const Phys* phs, const Sweep* sws, int count, int tiles, int threads,
                                    size_t smem, cudaStream_t st) {
  static int attr_dev = -1;
  int dev = 0;
  cudaGetDevice(&dev);
  if (attr_dev != dev) {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, k_sweep_batch<R, AX, EPT, GEN>);
    if (e != cudaSuccess) return e;
    int optin = 0;
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_sweep_batch<R, AX, EPT, GEN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             optin - (int)fa.sharedSizeBytes);
    if (e != cudaSuccess) return e;
    attr_dev = dev;
  }
  k_sweep_batch<R, AX, EPT, GEN><<<dim3(tiles, count), threads, smem, st>>>(phs, sws);
  return cudaGetLastError();
}

template <typename R>
cudaError_t launch_sweep_batch(int ax, bool gen, const Phys* phs, const Sweep* sws, int count, int tiles,
                               int threads, size_t smem, cudaStream_t st) {
  if (gen) {
    if (ax == AX_Z) return launch_batch_one<R, AX_Z, 8, true>(phs, sws, count, tiles, threads, smem, st);
    if (ax == AX_Y) return launch_batch_one<R, AX_Y, 8, true>(phs, sws, count, tiles, threads, smem, st);
    return launch_batch_one<R, AX_X, 8, true>(phs, sws, count, tiles, threads, smem, st);
  }
  if (ax == AX_Z) return launch_batch_one<R, AX_Z, 16, false>(phs, sws, count, tiles, threads, smem, st);
  if (ax == AX_Y) return launch_batch_one<R, AX_Y, 16, false>(phs, sws, count, tiles, threads, smem, st);
  return launch_batch_one<R, AX_X, 16, false>(phs, sws, count, tiles, threads, smem, st);
}

}  // namespace gpe
