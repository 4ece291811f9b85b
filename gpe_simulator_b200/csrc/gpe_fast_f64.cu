// Register-resident sweeps, complex128.
#include "gpe_fast_impl.cuh"
template cudaError_t gpe::launch_fast<double>(int, int, const gpe::Phys&, const gpe::Sweep&,
                                              const gpe::FastOps&, cudaStream_t);
template cudaError_t gpe::launch_fast_batch<double>(int, int, const gpe::Phys*, const gpe::Sweep*, int,
                                                   const gpe::FastOps&, cudaStream_t);
