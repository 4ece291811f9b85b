// gpe_fast_impl.cuh -- launch wrappers of the register-resident sweeps for one precision.
#pragma once
#include "gpe_fast.cuh"
#include "gpe_sweep.h"
#include "gpe_tma.cuh"

namespace gpe {

// the kernel of (N, AX, R, MODE): explicit occupancy bounds where measured
template <int N, int AX, typename R, int MODE> constexpr auto fast_kernel() {
  constexpr int B = FastBounds<N, R, MODE>::value;
  if constexpr (B > 0) return &k_fast_occ<N, AX, R, MODE, B>;
  else return &k_fast<N, AX, R, MODE>;
}
template <int N, int AX, typename R, int MODE> constexpr auto fast_batch_kernel() {
  constexpr int B = FastBounds<N, R, MODE>::value;
  if constexpr (B > 0) return &k_fast_batch_occ<N, AX, R, MODE, B>;
  else return &k_fast_batch<N, AX, R, MODE>;
}

// Blocks of `kern` resident on the whole device at once (the L2 prefetch
// distance of a sweep: the tile the next block on an SM will take).
template <typename K>
static cudaError_t resident_blocks(K kern, int threads, size_t smem, int& out) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
  out = e == cudaSuccess ? sms * per_sm : 0;
  return e;
}

template <int N, int AX, typename R, int MODE>
static cudaError_t launch_fast_one(const Phys& ph, const Sweep& sw, const FastOps& op_in, cudaStream_t st) {
  constexpr int L = FastCfg<N, R>::L;
  constexpr int T = FastCfg<N, R>::T;
  const int tiles = AX == FZ ? N * N / L : N * (N / L);
  constexpr size_t smem = fast_smem_bytes<N, R>();
  constexpr auto kern = fast_kernel<N, AX, R, MODE>();
  static int attr_dev = -1, resident = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  if (attr_dev != dev) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) e = resident_blocks(kern, T, smem, resident);
    if (e != cudaSuccess) return e;
    attr_dev = dev;
  }
  FastOps op = op_in;
  op.pf = resident < tiles ? resident : 0;
  if (!op.pdl) {
    kern<<<tiles, T, smem, st>>>(ph, sw, op);
    return cudaGetLastError();
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)tiles);
  cfg.blockDim = dim3(T);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, ph, sw, op);
}

template <int N, typename R>
cudaError_t launch_fast_n(int ax, const Phys& ph, const Sweep& sw, const FastOps& op, cudaStream_t st) {
  switch (op.mode) {
    case FM_Z1: return launch_fast_one<N, FZ, R, FM_Z1>(ph, sw, op, st);
    case FM_Z2: return launch_fast_one<N, FZ, R, FM_Z2>(ph, sw, op, st);
    case FM_Z21: return launch_fast_one<N, FZ, R, FM_Z21>(ph, sw, op, st);
    case FM_XKIN: return launch_fast_one<N, FX, R, FM_XKIN>(ph, sw, op, st);
    case FM_DIAGR: return launch_fast_one<N, FZ, R, FM_DIAGR>(ph, sw, op, st);
    case FM_DIAGK: return launch_fast_one<N, FX, R, FM_DIAGK>(ph, sw, op, st);
    default: break;
  }
  if (ax == FZ) return launch_fast_one<N, FZ, R, FM_PLAIN>(ph, sw, op, st);
  if (ax == FY) return launch_fast_one<N, FY, R, FM_PLAIN>(ph, sw, op, st);
  return launch_fast_one<N, FX, R, FM_PLAIN>(ph, sw, op, st);
}

template <int N, int AX, typename R, int MODE>
static cudaError_t launch_fastb_one(const Phys* phs, const Sweep* sws, int count, const FastOps& op_in,
                                    cudaStream_t st) {
  constexpr int L = FastCfg<N, R>::L;
  constexpr int T = FastCfg<N, R>::T;
  const int tiles = AX == FZ ? N * N / L : N * (N / L);
  constexpr size_t smem = fast_smem_bytes<N, R>();
  constexpr auto kern = fast_batch_kernel<N, AX, R, MODE>();
  static int attr_dev = -1, resident = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  if (attr_dev != dev) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) e = resident_blocks(kern, T, smem, resident);
    if (e != cudaSuccess) return e;
    attr_dev = dev;
  }
  // blocks run x (tile) fastest, so the next block on an SM takes tile + resident
  // of the same instance while the instance has that many tiles left
  FastOps op = op_in;
  op.pf = resident < tiles ? resident : 0;
  kern<<<dim3(tiles, count), T, smem, st>>>(phs, sws, op);
  return cudaGetLastError();
}

template <int N, typename R>
cudaError_t launch_fastb_n(int ax, const Phys* phs, const Sweep* sws, int count, const FastOps& op,
                                  cudaStream_t st) {
  switch (op.mode) {
    case FM_Z1: return launch_fastb_one<N, FZ, R, FM_Z1>(phs, sws, count, op, st);
    case FM_Z2: return launch_fastb_one<N, FZ, R, FM_Z2>(phs, sws, count, op, st);
    case FM_Z21: return launch_fastb_one<N, FZ, R, FM_Z21>(phs, sws, count, op, st);
    case FM_XKIN: return launch_fastb_one<N, FX, R, FM_XKIN>(phs, sws, count, op, st);
    case FM_DIAGR: return launch_fastb_one<N, FZ, R, FM_DIAGR>(phs, sws, count, op, st);
    case FM_DIAGK: return launch_fastb_one<N, FX, R, FM_DIAGK>(phs, sws, count, op, st);
    default: break;
  }
  if (ax == FZ) return launch_fastb_one<N, FZ, R, FM_PLAIN>(phs, sws, count, op, st);
  if (ax == FY) return launch_fastb_one<N, FY, R, FM_PLAIN>(phs, sws, count, op, st);
  return launch_fastb_one<N, FX, R, FM_PLAIN>(phs, sws, count, op, st);
}

// Persistent TMA-staged y/x sweep: as many blocks as are resident, each taking an
// equal share of the tiles (ceil(tiles / resident) tiles per block).
template <int N, int AX>
static cudaError_t launch_tma_one(const Phys& ph, const Sweep& sw, const FastOps& op, const CUtensorMap& map,
                                  cudaStream_t st) {
  constexpr int T = FastCfg<N, float>::T;
  constexpr int NT = N * (N / FastCfg<N, float>::L);
  constexpr size_t smem = TmaCfg<N>::SMEM;
  constexpr auto kern = &k_tma_plain<N, AX>;
  static int attr_dev = -1, resident = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  if (attr_dev != dev) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0, sms = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, T, smem);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    resident = (per_sm > 0 ? per_sm : 1) * sms;
    attr_dev = dev;
  }
  const int per_block = (NT + resident - 1) / resident;
  const int grid = (NT + per_block - 1) / per_block;
  if (!op.pdl) {
    kern<<<grid, T, smem, st>>>(ph, sw, op, map);
    return cudaGetLastError();
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(T);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, ph, sw, op, map);
}

template <int N>
cudaError_t launch_tma_n(int ax, const Phys& ph, const Sweep& sw, const FastOps& op, const CUtensorMap& map,
                         cudaStream_t st) {
  if (op.mode != FM_PLAIN) return cudaErrorInvalidValue;
  if (ax == FY) return launch_tma_one<N, FY>(ph, sw, op, map, st);
  if (ax == FX) return launch_tma_one<N, FX>(ph, sw, op, map, st);
  return cudaErrorInvalidValue;
}

// Persistent plane-fused launch: one block per resident slot.  The scheduling
// window is the smallest divisor W of N for which a producer task is handed out
// at least AHEAD x (tickets in flight = 2 per block) tickets before its
// consumers; the producer-consumer distance is stages x W x N/L tickets.
template <int N, typename R, int MZ>
static cudaError_t launch_plane_one(const Phys& ph, const Sweep& sw, PlaneJob job, cudaStream_t st) {
  constexpr int L = FastCfg<N, R>::L;
  constexpr int T = FastCfg<N, R>::T;
  constexpr int TPP = N / L;
  constexpr size_t smem = fast_smem_bytes<N, R>();
  static int attr_dev = -1, resident = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  if (attr_dev != dev) {
    cudaError_t e = cudaFuncSetAttribute(k_plane<N, R, MZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0, sms = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_plane<N, R, MZ>, T, smem);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    resident = (per_sm > 0 ? per_sm : 1) * sms;
    attr_dev = dev;
  }
  if (job.nstage < 1 || job.nstage > 3 || job.zstage < 0 || job.zstage >= job.nstage) return cudaErrorInvalidValue;
#ifndef GPE_PLANE_AHEAD
#define GPE_PLANE_AHEAD 1
#endif
  int w = N;
  for (int c = 1; c <= N; ++c)
    if (N % c == 0 && c * TPP * job.nstage >= GPE_PLANE_AHEAD * 2 * resident) { w = c; break; }
  job.window = w;
  const int tasks = N * TPP * job.nstage;
  const int grid = resident < tasks ? resident : tasks;
  k_plane<N, R, MZ><<<grid, T, smem, st>>>(ph, sw, job);
  return cudaGetLastError();
}

template <int N, typename R>
cudaError_t launch_plane_n(int mz, const Phys& ph, const Sweep& sw, PlaneJob job, cudaStream_t st) {
  switch (mz) {
    case FM_Z1: return launch_plane_one<N, R, FM_Z1>(ph, sw, job, st);
    case FM_Z2: return launch_plane_one<N, R, FM_Z2>(ph, sw, job, st);
    case FM_Z21: return launch_plane_one<N, R, FM_Z21>(ph, sw, job, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace gpe
