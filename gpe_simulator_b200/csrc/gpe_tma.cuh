// gpe_tma.cuh -- y/x sweeps whose pencils are staged by the Tensor Memory
// Accelerator (complex64, n = 128, 256).
//
// A y (or x) tile is L = 16 lines of n points along the transform axis at 16
// consecutive z: n rows of 128 contiguous bytes, one 3-D TMA box {16, n, 1}
// (x tiles: {16, 1, n}) of 16 n complex64.  The kernel is persistent: each block
// walks the tiles blockIdx.x, blockIdx.x + gridDim.x, ... through two
// shared-memory stages.  One elected thread issues `cp.async.bulk.tensor` for the
// tile after next as soon as a stage is free, so the next pencil streams in
// while the current one is transformed; completion is signalled on the stage's
// mbarrier (transaction count = tile bytes).  The stage doubles as the FFT's
// exchange buffer (the y/x exchange [k2][lane][L] has exactly 16 n entries), so
// a block holds 2 tiles + twiddles (68 KB at n = 256): 3 blocks per SM.  The
// stages start on a 128-byte boundary of shared memory (rule of tiled TMA copies).
//
// Arithmetic is that of the register-resident sweep (same FFT, same order of
// operations), so results are bit-identical to it; only the load path differs.
// Opt-in (sweep path 4): measured on B200 at 256^3 the staged y sweep takes the
// same 51 us as the plain-load one (both near the 45.7 us copy floor of 128-byte
// rows at a 2 KB stride), and a step is 4-5% slower because the persistent grid
// holds the SMs until its last tile, ending the programmatic overlap with the
// neighbouring sweeps.
// Every wait on an mbarrier is bounded (GPE_TMA_WAIT_NS of global time); on
// expiry the block records ST_TIMEOUT, issues no further copy, waits once more
// (bounded) for the copies it has in flight, and all its threads leave together.
// A copy that outlasts that second wait too can still land after the block has
// left; the status word reports the timeout either way.
#pragma once
#include <cuda.h>
#include "gpe_fast.cuh"

namespace gpe {

#ifndef GPE_TMA_WAIT_NS
#define GPE_TMA_WAIT_NS 2000000000ull   // 2 s
#endif

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// 3-D tiled bulk copy global -> shared of this CTA (no multicast), completion
// counted on `bar`.  c0 is the innermost (z) coordinate: a multiple of 16
// elements of 8 bytes, so the copy starts on a 16-byte boundary.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, unsigned long long* bar, int c0,
                                            int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(smem_addr(dst)), "l"((unsigned long long)map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(bar))
      : "memory");
}

// Wait (all threads) for phase `parity` of `bar`; true when it completed in time.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait(bar, parity))
    if (global_ns() - t0 > GPE_TMA_WAIT_NS) return false;
  return true;
}

template <int N> struct TmaCfg {
  static constexpr bool ok = N == 128 || N == 256;
  static constexpr int L = FastCfg<N, float>::L;
  static constexpr int TILE = L * N;                               // complex64 per tile
  static constexpr unsigned TILE_BYTES = (unsigned)TILE * 8u;
  static constexpr int TW_ENTRIES = N;                              // float4 each
  // stages (128-byte aligned: the TMA destination rule), twiddles, 2 mbarriers,
  // plus the slack that aligns the stages within the dynamic shared memory
  static constexpr size_t SMEM = 128 + 2 * (size_t)TILE_BYTES + (size_t)TW_ENTRIES * 16 + 2 * 8;
};

// TMA coordinates (z, y, x) of tile `tile` of axis AX (FastTile's numbering).
template <int N, int AX>
__device__ __forceinline__ void tma_coords(int tile, int& c0, int& c1, int& c2) {
  constexpr int TPR = N / TmaCfg<N>::L;
  const int row = tile / TPR, z0 = (tile % TPR) * TmaCfg<N>::L;
  c0 = z0;
  if (AX == FY) { c1 = 0; c2 = row; }
  else { c1 = row; c2 = 0; }
}

// Plain FFT sweep (op.inv1: inverse; op.invm: times 1/M) along y or x.
template <int N, int AX>
__device__ __forceinline__ void tma_plain_body(const Phys& ph, const Sweep& sw, const FastOps& op,
                                               const CUtensorMap* map) {
  using R = float;
  using C = typename Cx<R>::T;
  using TW = typename TwE<R>::T;
  constexpr int L = FastCfg<N, R>::L;
  constexpr int T = FastCfg<N, R>::T;
  constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
  constexpr int EPT = FastCfg<N, R>::V;
  constexpr int S1 = FastCfg<N, R>::Q1, S2 = FastCfg<N, R>::Q2;
  constexpr int TILE = TmaCfg<N>::TILE;
  constexpr int NT = N * (N / L);
  static_assert(TmaCfg<N>::ok && (AX == FY || AX == FX), "TMA sweeps: complex64 y/x tiles, n = 128, 256");
  static_assert(L * 8 % 16 == 0, "TMA box rows must be multiples of 16 bytes");
  griddep_launch_dependents();
  // dynamic shared memory only (no static variables), its start rounded up to
  // 128 bytes: only 16-byte alignment of the dynamic region is guaranteed
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* base = smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u);
  C* stage0 = (C*)base;
  TW* t1 = (TW*)(base + 2 * (size_t)TmaCfg<N>::TILE_BYTES);
  unsigned long long* bar = (unsigned long long*)(t1 + TmaCfg<N>::TW_ENTRIES);
  // self-check of the copy rules (destination 128-byte aligned, barrier 8-byte
  // aligned, both inside the launch's shared memory, tensor map 64-byte
  // aligned); uniform over the block
  if ((smem_addr(stage0) & 127u) || (smem_addr(bar) & 7u) || ((unsigned long long)map & 63u) ||
      (size_t)((unsigned char*)(bar + 2) - smem_raw) > TmaCfg<N>::SMEM) {
    if (threadIdx.x == 0) atomicOr(sw.status, ST_LAYOUT);
    return;
  }

  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init_fence();
  }
  // twiddle tables (plan constants): built before the dependency wait
  {
    const C* gh = (const C*)sw.tw;
    const C* gl = (const C*)sw.tw_lo;
    for (int q = threadIdx.x; q < N; q += T) {
      const int k2 = q / N1, n1 = q % N1;   // t1[k2*N1 + n1] = W^(n1*k2)
      const int e = n1 * k2;
      t1[q] = make_float4(gh[e].x, gh[e].y, gl[e].x, gl[e].y);
    }
  }
  __syncthreads();  // barriers initialised, twiddles visible
  griddep_wait();   // psi comes from the previous sweep

  const int first = blockIdx.x, stride = gridDim.x;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int tile = first + k * stride;
      if (tile < NT) {
        int c0, c1, c2;
        tma_coords<N, AX>(tile, c0, c1, c2);
        mbar_expect_tx(&bar[k], TmaCfg<N>::TILE_BYTES);
        tma_load_3d(stage0 + k * TILE, map, &bar[k], c0, c1, c2);
      }
    }
  }
  const bool inv = op.inv1 != 0;
  int it = 0;
  for (int tile = first; tile < NT; tile += stride, ++it) {
    const int s = it & 1;
    C* stage = stage0 + s * TILE;
    const bool done = mbar_wait_bounded(&bar[s], (unsigned)(it >> 1) & 1u);
    if (__syncthreads_or(!done)) {
      if (threadIdx.x == 0) atomicOr(sw.status, ST_TIMEOUT);
      // Copies still in flight write into this block's shared memory, which the
      // SM may hand to another block once this one exits: issue nothing more
      // and wait once more (bounded) for the late copy of this stage and for
      // the prefetch of the next tile into the other stage, if one was issued.
      mbar_wait_bounded(&bar[s], (unsigned)(it >> 1) & 1u);
      if (tile + stride < NT) mbar_wait_bounded(&bar[s ^ 1], (unsigned)((it + 1) >> 1) & 1u);
      __syncthreads();
      return;
    }
    // registers in layout (N1 lanes, N2 values); the staged box is [m][l]
    C v[EPT];
#pragma unroll
    for (int q = 0; q < S1; ++q) {
      if (!slot_ok<N, R, N1, S1>(q)) break;
      int l, lane;
      slot<AX, L, T>(threadIdx.x + q * T, N1, l, lane);
#pragma unroll
      for (int b = 0; b < N2; ++b) {
        const C x = stage[(lane + N1 * b) * L + l];
        v[q * N2 + b] = inv ? conj_<R>(x) : x;
      }
    }
    __syncthreads();  // the stage becomes the exchange buffer
    // the exchange in the stage, fenced against the copy that refills it
    fft_2phase<N, N1, N2, AX, R, S1, S2, EPT, true>(v, stage, t1);  // ends with a block barrier
    if (threadIdx.x == 0) {
      const int next = tile + 2 * stride;
      if (next < NT) {
        int c0, c1, c2;
        tma_coords<N, AX>(next, c0, c1, c2);
        mbar_expect_tx(&bar[s], TmaCfg<N>::TILE_BYTES);
        tma_load_3d(stage, map, &bar[s], c0, c1, c2);
      }
    }
    if (inv) conj_all(v);
    if (op.invm) scale_all(v, (R)ph.inv_m);
    const FastTile<N, AX, R> tl(tile);
    fast_store<N, AX, R, N2, N1, S2>(v, tl, (C*)sw.dst);
  }
}

template <int N, int AX>
__global__ void __launch_bounds__(FastCfg<N, float>::T, FastCfg<N, float>::T >= 512 ? 1 : 3)
    k_tma_plain(Phys ph, Sweep sw, FastOps op, const __grid_constant__ CUtensorMap map) {
  tma_plain_body<N, AX>(ph, sw, op, &map);
}

}  // namespace gpe
