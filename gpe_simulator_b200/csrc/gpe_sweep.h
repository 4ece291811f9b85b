// gpe_sweep.h -- host entry points of the sweep kernels (one translation unit per precision).
#pragma once
#include <cuda_runtime.h>
#include "gpe_kernels.cuh"

namespace gpe {

// Launch one sweep along axis `ax` (AX_Z/AX_Y/AX_X).  `gen` selects the kernel
// family that also carries the odd-prime radices 7, 11, 13.
template <typename R>
cudaError_t launch_sweep(int ax, bool gen, const Phys& ph, const Sweep& sw, int tiles, int threads,
                         size_t smem, cudaStream_t st);

// Batched launch: grid (tiles, count), instance i reads phs[i] and sws[i] (device arrays).
template <typename R>
cudaError_t launch_sweep_batch(int ax, bool gen, const Phys* phs, const Sweep* sws, int count, int tiles,
                               int threads, size_t smem, cudaStream_t st);

}  // namespace gpe
