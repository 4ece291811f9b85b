// Register-resident sweeps, n = 512, float (complex64 only).
#include "gpe_fast_impl.cuh"
template cudaError_t gpe::launch_fast_n<512, float>(int, const gpe::Phys&, const gpe::Sweep&,
                                                 const gpe::FastOps&, cudaStream_t);
template cudaError_t gpe::launch_fastb_n<512, float>(int, const gpe::Phys*, const gpe::Sweep*, int,
                                                  const gpe::FastOps&, cudaStream_t);
