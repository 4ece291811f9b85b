// Sweep kernels, complex128.
#include "gpe_sweep_impl.cuh"
template cudaError_t gpe::launch_sweep<double>(int, bool, const gpe::Phys&, const gpe::Sweep&, int, int,
                                               size_t, cudaStream_t);
template cudaError_t gpe::launch_sweep_batch<double>(int, bool, const gpe::Phys*, const gpe::Sweep*, int, int,
                                                     int, size_t, cudaStream_t);
