// Dispatch of the register-resident sweeps by grid size (one translation unit per
// size and precision holds the kernels: gpe_fast_<prec>_<n>.cu).
#include <cuda.h>
#include "gpe_fast.cuh"

namespace gpe {

template <int N, typename R>
cudaError_t launch_fast_n(int ax, const Phys& ph, const Sweep& sw, const FastOps& op, cudaStream_t st);
template <int N, typename R>
cudaError_t launch_fastb_n(int ax, const Phys* phs, const Sweep* sws, int count, const FastOps& op,
                           cudaStream_t st);

template <int N, typename R>
cudaError_t launch_plane_n(int mz, const Phys& ph, const Sweep& sw, PlaneJob job, cudaStream_t st);

#define GPE_FAST_SIZES(X) X(32) X(48) X(64) X(96) X(128) X(160) X(256)

template <typename R>
cudaError_t launch_fast(int n, int ax, const Phys& ph, const Sweep& sw, const FastOps& op, cudaStream_t st) {
  switch (n) {
#define GPE_CASE(NN) case NN: return launch_fast_n<NN, R>(ax, ph, sw, op, st);
    GPE_FAST_SIZES(GPE_CASE)
#undef GPE_CASE
    case 512:
      if constexpr (sizeof(R) == 4) return launch_fast_n<512, float>(ax, ph, sw, op, st);
      return cudaErrorInvalidValue;
    default: return cudaErrorInvalidValue;
  }
}

template <typename R>
cudaError_t launch_fast_batch(int n, int ax, const Phys* phs, const Sweep* sws, int count, const FastOps& op,
                              cudaStream_t st) {
  switch (n) {
#define GPE_CASE(NN) case NN: return launch_fastb_n<NN, R>(ax, phs, sws, count, op, st);
    GPE_FAST_SIZES(GPE_CASE)
#undef GPE_CASE
    case 512:
      if constexpr (sizeof(R) == 4) return launch_fastb_n<512, float>(ax, phs, sws, count, op, st);
      return cudaErrorInvalidValue;
    default: return cudaErrorInvalidValue;
  }
}

template <int N>
cudaError_t launch_tma_n(int ax, const Phys& ph, const Sweep& sw, const FastOps& op, const CUtensorMap& map,
                         cudaStream_t st);

// TMA-staged plain y/x sweeps: complex64, n = 128 and 256
cudaError_t launch_fast_tma(int n, int ax, const Phys& ph, const Sweep& sw, const FastOps& op,
                            const CUtensorMap& map, cudaStream_t st) {
  switch (n) {
    case 128: return launch_tma_n<128>(ax, ph, sw, op, map, st);
    case 256: return launch_tma_n<256>(ax, ph, sw, op, map, st);
    default: return cudaErrorInvalidValue;
  }
}

// plane-fused y/z sweeps: complex64, n = 128 and 256
template <typename R>
cudaError_t launch_plane(int n, int mz, const Phys& ph, const Sweep& sw, const PlaneJob& job, cudaStream_t st) {
  if (sizeof(R) != 4) return cudaErrorInvalidValue;
  switch (n) {
    case 128: return launch_plane_n<128, float>(mz, ph, sw, job, st);
    case 256: return launch_plane_n<256, float>(mz, ph, sw, job, st);
    default: return cudaErrorInvalidValue;
  }
}

template cudaError_t launch_plane<float>(int, int, const Phys&, const Sweep&, const PlaneJob&, cudaStream_t);
template cudaError_t launch_fast<float>(int, int, const Phys&, const Sweep&, const FastOps&, cudaStream_t);
template cudaError_t launch_fast<double>(int, int, const Phys&, const Sweep&, const FastOps&, cudaStream_t);
template cudaError_t launch_fast_batch<float>(int, int, const Phys*, const Sweep*, int, const FastOps&,
                                              cudaStream_t);
template cudaError_t launch_fast_batch<double>(int, int, const Phys*, const Sweep*, int, const FastOps&,
                                               cudaStream_t);

}  // namespace gpe
