// Register-resident sweeps, complex128.
#include "gpe_fast_impl.cuh"
template cudaError_t gpe::launch_fast<double>(int, int, const gpe::Phys&, const gpe::Sweep&,
                                              const gpe::FastOps&, cudaStream_t);
