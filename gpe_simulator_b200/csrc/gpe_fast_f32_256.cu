// Register-resident sweeps, n = 256, float.
#include "gpe_fast_impl.cuh"
template cudaError_t gpe::launch_fast_n<256, float>(int, const gpe::Phys&, const gpe::Sweep&,
                                                 const gpe::FastOps&, cudaStream_t);
template cudaError_t gpe::launch_fastb_n<256, float>(int, const gpe::Phys*, const gpe::Sweep*, int,
                                                  const gpe::FastOps&, cudaStream_t);
template cudaError_t gpe::launch_plane_n<256, float>(int, const gpe::Phys&, const gpe::Sweep&, gpe::PlaneJob,
                                                     cudaStream_t);
template cudaError_t gpe::launch_tma_n<256>(int, const gpe::Phys&, const gpe::Sweep&, const gpe::FastOps&,
                                          const CUtensorMap&, cudaStream_t);
