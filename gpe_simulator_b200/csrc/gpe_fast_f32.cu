// Register-resident sweeps, complex64.
#include "gpe_fast_impl.cuh"
template cudaError_t gpe::launch_fast<float>(int, int, const gpe::Phys&, const gpe::Sweep&,
                                             const gpe::FastOps&, cudaStream_t);
template cudaError_t gpe::launch_fast_batch<float>(int, int, const gpe::Phys*, const gpe::Sweep*, int,
                                                   const gpe::FastOps&, cudaStream_t);
