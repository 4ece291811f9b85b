// Sweep kernels, complex64.
#include "gpe_sweep_impl.cuh"
template cudaError_t gpe::launch_sweep<float>(int, bool, const gpe::Phys&, const gpe::Sweep&, int, int,
                                              size_t, cudaStream_t);
template cudaError_t gpe::launch_sweep_batch<float>(int, bool, const gpe::Phys*, const gpe::Sweep*, int, int,
                                                    int, size_t, cudaStream_t);
