// gpe_fast.cuh -- register-resident sweep kernels for N = 32, 64, 128, 256 (sm_100a).
//
// A line of length N = N1*N2 is transformed in two register phases with one
// shared-memory exchange between them (the "four-step" split):
//   phase 1: thread n1 (< N1) holds x[n1 + N1*n2], n2 < N2, and computes
//            Y[n1][k2] = DFT_N2(x[n1 + N1*.])[k2] * W_N^(n1*k2);
//   exchange through shared memory;
//   phase 2: thread k2 (< N2) holds Y[.][k2] and computes
//            X[k2 + N2*k1] = DFT_N1(Y[.][k2])[k1].
// Values come straight from HBM into phase-1 registers and leave from phase-2
// registers, so an FFT costs one shared-memory round trip.  The output layout
// (thread k2 holds k2 + N2*k1) is the input layout of the same algorithm with
// N1 and N2 swapped, so an inverse transform can start from the forward's
// registers with no exchange (the kinetic sweep: forward, kinetic phase,
// inverse).  Inverses are conj(FFT(conj(x))).
//
// Tiles: Z = L consecutive z-lines (contiguous in memory; consecutive lanes
// walk along the line), P = L adjacent lines of the y or x axis (consecutive
// lanes walk across lines, 128-byte rows).  Pointwise work (renormalisation,
// half-steps, 1/M, kinetic phase, norm partials) runs on the registers.
#pragma once
#include <type_traits>

#include "gpe_kernels.cuh"

namespace gpe {

// N = N1*N2: phase 1 runs DFT_N2 on N1 lanes, phase 2 DFT_N1 on N2 lanes.
template <int N> struct Split;
template <> struct Split<32>  { static constexpr int N1 = 4,  N2 = 8;  };
template <> struct Split<48>  { static constexpr int N1 = 6,  N2 = 8;  };
template <> struct Split<64>  { static constexpr int N1 = 8,  N2 = 8;  };
template <> struct Split<96>  { static constexpr int N1 = 12, N2 = 8;  };
template <> struct Split<128> { static constexpr int N1 = 8,  N2 = 16; };
template <> struct Split<160> { static constexpr int N1 = 10, N2 = 16; };
template <> struct Split<256> { static constexpr int N1 = 16, N2 = 16; };
// n = 512: three radix-8 phases over 64 lanes (fft_3phase); N1 = 64 lanes and
// N2 = 8 values per slot in every layout
template <> struct Split<512> { static constexpr int N1 = 64, N2 = 8; };

__host__ __device__ constexpr int cdiv(int a, int b) { return (a + b - 1) / b; }

// Lines per tile L (128-byte rows for y/x tiles) and threads per
// block T.  The layout (N1 lanes, N2 values) has P1 = L*N1 slots, (N2 lanes, N1
// values) has P2 = L*N2; a thread holds Q1 (resp. Q2) slots, some threads idle in
// one phase when P1 != P2 do not divide evenly.
// lines per tile of the register-resident sweeps (host and device): 16 for
// complex64 (128-byte rows in y/x tiles), 8 for complex128 (also 128 bytes).
// At n = 512 (complex64 only) 16 lines take 512 threads; measured against 8
// lines (256 threads, 64-byte rows): 291 -> 312 steps/s at 512^3, the gain
// being in the overlap of programmatically launched sweeps (per-launch times
// alike).  32 lines at n = 256 (512 threads) measured 3141 vs 4150 steps/s:
// the fused sweeps drop to 16 resident warps per SM (Z21 113 vs 84 us); 32
// lines at n = 128 (256 threads) 26.3k vs 28.1k steps/s at 128^3 and the same
// batched throughput.
__host__ __device__ constexpr int fast_lines(int n, int real_bytes) {
  return n == 512 ? 16 : (real_bytes == 4 ? 16 : 8);
}

template <int N, typename R> struct FastCfg {
  static constexpr int L = fast_lines(N, (int)sizeof(R));
  static constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
  // three-phase transform (n = 512): the layout (N1 lanes, N2 values) in and out
  static constexpr bool THREE = N == 512;
  static constexpr int P1 = L * N1, P2 = THREE ? P1 : L * N2;
  static constexpr bool POW2 = (N & (N - 1)) == 0 && N <= 512;
  // power-of-two sizes: 16 values per thread; other sizes: one slot per thread per phase
  static constexpr int T0 = POW2 ? L * N / 16 : cdiv(P1 > P2 ? P1 : P2, 32) * 32;
  static constexpr int T = T0 < 32 ? 32 : T0;
  static constexpr int Q1 = cdiv(P1, T), Q2 = cdiv(P2, T);
  // registers (complex) per thread
  static constexpr int V = THREE ? Q1 * N2 : (Q1 * N2 > Q2 * N1 ? Q1 * N2 : Q2 * N1);
};

enum : int { FZ = 0, FY = 1, FX = 2 };

// shared exchange buffer (complex elements) covering both split orders and tile kinds
template <int N, typename R> __host__ __device__ constexpr int fast_exchange_elems() {
  return FastCfg<N, R>::L * (N + (Split<N>::N1 > Split<N>::N2 ? Split<N>::N1 : Split<N>::N2));
}

// runtime options of a fast sweep (uniform per launch)
struct FastOps {
  int mode;         // FM_* (selects the kernel)
  int inv1;         // FM_PLAIN: inverse transform
  int invm;         // FM_PLAIN: multiply by 1/M
  int scale;        // FM_Z1: apply the pending renormalisation
  int norm;         // FM_Z2: norm partials and renormalisation scale
  int pdl;          // host: launch as a programmatic dependent of the previous sweep
  int pf;           // tiles ahead whose lines a block prefetches into L2 (0 = none): the
                    // tile the block that follows it on the SM will process
};

// Programmatic dependent launch: a sweep lets the next one start (its blocks
// then build their shared-memory tables while this sweep's last wave runs) and
// waits for the previous sweep's results before touching psi.  Without a
// programmatic launch the wait returns at once.
__device__ __forceinline__ void griddep_launch_dependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Order this thread's generic-proxy shared-memory accesses before later
// async-proxy (TMA) accesses of the same bytes.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// per-tile table bytes (kx, kyz, kx2, kyz2, vz, c1, c2, c12), rounded to 16
template <int N, typename R> __host__ __device__ constexpr size_t fast_tables_bytes() {
  return (((size_t)(N + FastCfg<N, R>::L) * (16 + 8) + (size_t)(N + 3 * FastCfg<N, R>::L) * sizeof(R)) + 15)
         / 16 * 16;
}

// the same at run time (host): the shell histogram of a diagnostic x sweep lives
// in the tables region, so it holds at most this many bytes of bins
inline size_t fast_tables_bytes_rt(int n, int real_bytes) {
  const int L = fast_lines(n, real_bytes);
  return (((size_t)(n + L) * (16 + 8) + (size_t)(n + 3 * L) * real_bytes) + 15) / 16 * 16;
}

// shared memory of a fast sweep (bytes)
template <int N, typename R> __host__ __device__ constexpr size_t fast_smem_bytes() {
  return (size_t)(2 * N) * sizeof(typename Cx<R>::T)
         + (size_t)FastCfg<N, R>::L * (N + (Split<N>::N1 > Split<N>::N2 ? Split<N>::N1 : Split<N>::N2))
               * sizeof(typename Cx<R>::T)
         + 32 * 4 * 16                                          /* Acc reduction */
         + fast_tables_bytes<N, R>()
         + (FastCfg<N, R>::THREE ? (size_t)64 * sizeof(typename TwE<R>::T)          /* t2: W_64 */
            : Split<N>::N1 == Split<N>::N2 ? 0 : (size_t)(2 * N) * sizeof(typename Cx<R>::T));  /* t2 */
}

template <int N, int AX, typename R>
struct FastTile {
  static constexpr int L = FastCfg<N, R>::L;
  long long base;    // global index of (line 0, element 0)
  long long nstride; // stride along the transform axis
  long long lstride; // stride between lines
  int a0, b0;        // Z: first line g; Y: (x, z0); X: (y, z0)
  __device__ __forceinline__ FastTile(int tile) {
    if (AX == FZ) {
      a0 = tile * L; b0 = 0;
      base = (long long)a0 * N; nstride = 1; lstride = N;
    } else {
      constexpr int tpr = N / L;
      const int row = tile / tpr, z0 = (tile % tpr) * L;
      a0 = row; b0 = z0;
      lstride = 1;
      if (AX == FY) { base = (long long)row * N * N + z0; nstride = N; }
      else { base = (long long)row * N + z0; nstride = (long long)N * N; }
    }
  }
  __device__ __forceinline__ void coords(int l, int m, int& i, int& j, int& k) const {
    if (AX == FZ) { const int g = a0 + l; i = g / N; j = g % N; k = m; }
    else if (AX == FY) { i = a0; j = m; k = b0 + l; }
    else { i = m; j = a0; k = b0 + l; }
  }
  __device__ __forceinline__ long long gidx(int l, int m) const { return base + l * lstride + (long long)m * nstride; }
};

// Slot s of thread t (gs = t + s*TT) in a phase with `per` lanes per line: Z tiles
// walk along the line (lane fastest), P tiles across lines (line fastest).  Z
// tiles of one warp per line (TT = 32 LL) with more than 32 lanes give each
// thread lanes t%32 + 32 s of line t/32, so that a line stays in its warp.
template <int AX, int LL, int TT>
__device__ __forceinline__ void slot(int gs, int per, int& l, int& lane) {
  if (AX == FZ) {
    if (TT == 32 * LL && per > 32) { const int t = gs % TT; l = t >> 5; lane = (t & 31) + 32 * (gs / TT); }
    else { lane = gs % per; l = gs / per; }
  } else {
    l = gs % LL; lane = gs / LL;
  }
}

// One forward FFT of every line of the tile, A = lanes in phase 1 (values A-strided),
// B = values per lane in phase 1.  In: v[s][b] = x[lane_s + A*b] of line l_s (phase-1
// slots).  Out: v[s][a] = X[lane_s + B*a] (phase-2 slots with B lanes per line).
template <int N, int A, int B, int AX, typename R, int QA, int QB, int V, bool ASYNC_NEXT = false, bool TAIL = true>
__device__ __forceinline__ void fft_2phase(typename Cx<R>::T (&v)[V], typename Cx<R>::T* ex,
                                           const typename TwE<R>::T* tw) {
  // In: QA slots of (A lanes, B values), slot s holding x[lane + A*b] in v[s*B + b].
  // Out: QB slots of (B lanes, A values), slot s holding X[lane + B*a] in v[s*A + a].
  // tw: 2-D twiddle table of this split, tw[k2*A + lane] = W_N^(lane*k2) ({hi, lo}
  // for complex64): consecutive lanes read consecutive entries.
  // ASYNC_NEXT: the exchange buffer is overwritten by a TMA copy after the final
  // barrier, so each thread fences its exchange accesses against the async proxy.
  // TAIL: end with a barrier that frees the exchange buffer for a next transform;
  // the last transform of a sweep leaves it out (nothing reuses the buffer).
  using C = typename Cx<R>::T;
  constexpr int L = FastCfg<N, R>::L;
  constexpr int T = FastCfg<N, R>::T;
  static_assert(QA * B <= V && QB * A <= V, "register array too small");
  // Z tiles with A == B lanes per line in both phases and one slot per thread:
  // every line is owned by the same warp in both phases (32/A lines per warp)
  // and its exchange rows are its own, so a warp barrier suffices.
  constexpr bool WARP_LOCAL = AX == FZ && A == B && QA == 1 && QB == 1 && 32 % A == 0 && L * A == T;
#pragma unroll
  for (int s = 0; s < QA; ++s) {
    const int gs = threadIdx.x + s * T;
    if (QA * T > L * A && gs >= L * A) break;
    int l, lane;
    slot<AX, L, T>(gs, A, l, lane);
    C* x = v + s * B;
    Dft<B>::run(x, (const C*)nullptr, (const C*)nullptr, N / B);
#pragma unroll
    for (int k2 = 1; k2 < B; ++k2) x[k2] = tw_apply(x[k2], tw[k2 * A + lane]);
    // exchange layout: Z tiles [l][k2][A + 1] (odd pitch), P tiles [k2][lane][L]
#pragma unroll
    for (int k2 = 0; k2 < B; ++k2) {
      const int idx = AX == FZ ? (l * B + k2) * (A + 1) + lane : (k2 * A + lane) * L + l;
      ex[idx] = x[k2];
    }
  }
  if (WARP_LOCAL) __syncwarp(); else __syncthreads();
  // phase 2: lane k2 (< B) gathers Y[.][k2], DFT_A
#pragma unroll
  for (int s = 0; s < QB; ++s) {
    const int gs = threadIdx.x + s * T;
    if (QB * T > L * B && gs >= L * B) break;
    int l, k2;
    slot<AX, L, T>(gs, B, l, k2);
    C* x = v + s * A;
#pragma unroll
    for (int n1 = 0; n1 < A; ++n1) {
      const int idx = AX == FZ ? (l * B + k2) * (A + 1) + n1 : (k2 * A + n1) * L + l;
      x[n1] = ex[idx];
    }
    Dft<A>::run(x, (const C*)nullptr, (const C*)nullptr, N / A);
  }
  if (ASYNC_NEXT) fence_proxy_async_smem();
  if (TAIL) {
    if (WARP_LOCAL) __syncwarp(); else __syncthreads();
  }
}

// One forward FFT of every line of the tile for N = 8^3 (n = 512), in three
// radix-8 phases over 64 lanes per line.  In and out the registers are in
// layout (64 lanes, 8 values): slot s of lane p holds v[s][b] = x[p + 64 b] on
// entry and X[p + 64 k] on return, so the two transforms of a fused sweep need
// no change of layout between them.  Index split: n = p + 64 b with p = p1 + 8 p2,
// k = k3 + 8 k1 + 64 k2.
//   phase 1 (lane p):         DFT8 over b -> k3, times W_512^(p k3)     (twa[k3*64 + p])
//   phase 2 (role p1 + 8 k3): DFT8 over p2 -> k1, times W_64^(p1 k1)    (twb[k1*8 + p1])
//   phase 3 (role k3 + 8 k1): DFT8 over p1 -> k2; lane k3 + 8 k1 holds X[lane + 64 k2]
// Exchange layouts: Z tiles (a warp per line) rows of 72 elements per (line, k),
// the second exchange at 8 p1 + (k3 ^ p1) within its row, so that the 8-byte
// accesses of a half warp avoid bank conflicts in both directions; P tiles
// line-fastest, [k][role][l].  A thread's two slots are 32 lanes apart, so its
// p1 is the same in both: each W_64 twiddle is loaded once for the two.
template <int N, int AX, typename R, int Q, int V, bool TAIL = true>
__device__ __forceinline__ void fft_3phase(typename Cx<R>::T (&v)[V], typename Cx<R>::T* ex,
                                           const typename TwE<R>::T* twa, const typename TwE<R>::T* twb) {
  using C = typename Cx<R>::T;
  constexpr int L = FastCfg<N, R>::L;
  constexpr int T = FastCfg<N, R>::T;
  constexpr int RD = 8, A = 64;
  static_assert(N == RD * RD * RD && Q * RD <= V && Q * T == L * A, "three-phase layout");
  constexpr bool WARP_LOCAL = AX == FZ && T == 32 * L;
  auto e1 = [](int l, int k3, int p) { return AX == FZ ? (l * RD + k3) * 72 + p : (k3 * A + p) * L + l; };
  auto e2 = [](int l, int k3, int k1, int p1) {
    return AX == FZ ? (l * RD + k1) * 72 + 8 * p1 + (k3 ^ p1) : ((k1 * RD + k3) * RD + p1) * L + l;
  };
  auto sync = [] { if (WARP_LOCAL) __syncwarp(); else __syncthreads(); };
#pragma unroll
  for (int s = 0; s < Q; ++s) {
    int l, p;
    slot<AX, L, T>(threadIdx.x + s * T, A, l, p);
    C* x = v + s * RD;
    Dft<RD>::run(x, (const C*)nullptr, (const C*)nullptr, N / RD);
#pragma unroll
    for (int k3 = 1; k3 < RD; ++k3) x[k3] = tw_apply(x[k3], twa[k3 * A + p]);
#pragma unroll
    for (int k3 = 0; k3 < RD; ++k3) ex[e1(l, k3, p)] = x[k3];
  }
  sync();
#pragma unroll
  for (int s = 0; s < Q; ++s) {
    int l, q;
    slot<AX, L, T>(threadIdx.x + s * T, A, l, q);
    const int p1 = q & 7, k3 = q >> 3;
    C* x = v + s * RD;
#pragma unroll
    for (int p2 = 0; p2 < RD; ++p2) x[p2] = ex[e1(l, k3, p1 + RD * p2)];
  }
  sync();
  static_assert(T % (8 * L) == 0 || AX == FZ, "slots 32 lanes apart");
#pragma unroll
  for (int s = 0; s < Q; ++s) Dft<RD>::run(v + s * RD, (const C*)nullptr, (const C*)nullptr, N / RD);
  {
    int l0, q0;
    slot<AX, L, T>(threadIdx.x, A, l0, q0);
    const int p1 = q0 & 7;
#pragma unroll
    for (int k1 = 1; k1 < RD; ++k1) {
      const typename TwE<R>::T w = twb[k1 * RD + p1];
#pragma unroll
      for (int s = 0; s < Q; ++s) v[s * RD + k1] = tw_apply(v[s * RD + k1], w);
    }
  }
#pragma unroll
  for (int s = 0; s < Q; ++s) {
    int l, q;
    slot<AX, L, T>(threadIdx.x + s * T, A, l, q);
    const int p1 = q & 7, k3 = q >> 3;
#pragma unroll
    for (int k1 = 0; k1 < RD; ++k1) ex[e2(l, k3, k1, p1)] = v[s * RD + k1];
  }
  sync();
#pragma unroll
  for (int s = 0; s < Q; ++s) {
    int l, q;
    slot<AX, L, T>(threadIdx.x + s * T, A, l, q);
    const int k3 = q & 7, k1 = q >> 3;
    C* x = v + s * RD;
#pragma unroll
    for (int p1 = 0; p1 < RD; ++p1) x[p1] = ex[e2(l, k3, k1, p1)];
    Dft<RD>::run(x, (const C*)nullptr, (const C*)nullptr, N / RD);
  }
  if (TAIL) sync();   // frees the exchange buffer for a next transform
}

template <typename R>
__device__ __forceinline__ typename Cx<R>::T conj_(typename Cx<R>::T v) { return mk(v.x, -v.y); }

template <int EPT, typename C>
__device__ __forceinline__ void conj_all(C (&v)[EPT]) {
#pragma unroll
  for (int q = 0; q < EPT; ++q) v[q].y = -v[q].y;
}

template <int EPT, typename C, typename R>
__device__ __forceinline__ void scale_all(C (&v)[EPT], R f) {
#pragma unroll
  for (int q = 0; q < EPT; ++q) { v[q].x *= f; v[q].y *= f; }
}

enum : int { FM_PLAIN = 0, FM_Z1 = 1, FM_Z2 = 2, FM_Z21 = 3, FM_XKIN = 4, FM_DIAGR = 5, FM_DIAGK = 6 };

// sin(x) and cos(x) - 1 from their Taylor series (Horner, FP32), valid for
// |x| <= pi/4 where the first omitted terms (x^13/13!, x^14/14!) are below 1e-11;
// callers use sincosf for larger arguments.
__device__ __forceinline__ void sin_cosm1_series(float x, float& s, float& cm1) {
  {
    const float z = x * x;
    s = x * fmaf(z, fmaf(z, fmaf(z, fmaf(z, fmaf(z, -2.5052108385441720e-08f, 2.7557319223985888e-06f),
                                         -1.9841269841269841e-04f), 8.3333333333333333e-03f),
                         -1.6666666666666667e-01f), 1.0f);
    cm1 = z * fmaf(z, fmaf(z, fmaf(z, fmaf(z, fmaf(z, 2.0876756987868099e-09f, -2.7557319223985891e-07f),
                                           2.4801587301587302e-05f), -1.3888888888888889e-03f),
                           4.1666666666666667e-02f), -0.5f);
  }
}

// Short forms for |x| <= 1/8 (first omitted terms x^7/7!, x^8/8!: below 8e-10
// of the result), the common case of real-time steps.
__device__ __forceinline__ void sin_cosm1_tiny(float x, float& s, float& cm1) {
  const float z = x * x;
  s = x * fmaf(z, fmaf(z, 8.3333333333333333e-03f, -1.6666666666666667e-01f), 1.0f);
  cm1 = z * fmaf(z, fmaf(z, -1.3888888888888889e-03f, 4.1666666666666667e-02f), -0.5f);
}
__device__ __forceinline__ float expm1_tiny(float x) {
  return x * fmaf(x, fmaf(x, fmaf(x, fmaf(x, fmaf(x, 1.3888888888888889e-03f, 8.3333333333333333e-03f),
         4.1666666666666667e-02f), 1.6666666666666667e-01f), 0.5f), 1.0f);
}

// exp(x) - 1 from its Taylor series, valid for |x| <= 1/2 (first omitted term
// x^10/10! < 3e-10); callers use expm1f beyond.
__device__ __forceinline__ float expm1_series(float x) {
  {
    return x * fmaf(x, fmaf(x, fmaf(x, fmaf(x, fmaf(x, fmaf(x, fmaf(x, fmaf(x, 2.7557319223985891e-06f,
           2.4801587301587302e-05f), 1.9841269841269841e-04f), 1.3888888888888889e-03f), 8.3333333333333333e-03f),
           4.1666666666666667e-02f), 1.6666666666666667e-01f), 0.5f), 1.0f);
  }
}

// Per-tile tables in shared memory.
template <typename R>
struct FastTables {
  R* vz;          // [N] static potential along z (Z tiles)
  R* c1;          // [L] vx(i) + vy(j_l) + beam(i, j_l; t1)
  R* c2;          // [L] same at t2
  R* c12;         // [L] c1 + c2
  double2* kx;    // [N] kinetic factors along the transform axis (X tiles)
  double2* kyz;   // [L] kinetic factor of (j, k_l)
  double* kx2;    // [N] k^2 along x (cutoff)
  double* kyz2;   // [L] k_j^2 + k_kl^2
};

// two: the tables of the fused z sweep (c2, c12 at the second half-step's time).
// pre (real time, two half-steps as one rotation, no potential arrays): vz and
// c12 are stored already multiplied by dt (vz by dt, c12 by dt/2), so that the
// phase (2 vz + c12 + 2 beta |psi|^2) dt/2 is one add and one fma per point.
template <int N, typename R>
__device__ __forceinline__ void z_tables(const Phys& ph, const Sweep& sw, int a0, FastTables<R>& tb,
                                         bool two, bool pre = false) {
  constexpr int L = FastCfg<N, R>::L, T = FastCfg<N, R>::T;
  const R* vax = (const R*)ph.vax;
  const R h = (R)(ph.dt * 0.5), dt2 = h + h;
  for (int q = threadIdx.x; q < N; q += T) tb.vz[q] = pre ? vax[2 * N + q] * dt2 : vax[2 * N + q];
  if (threadIdx.x < L) {
    const int g = a0 + threadIdx.x, i = g / N, j = g % N;
    const R base = vax[i] + vax[N + j];
    R b1 = (R)0, b2 = (R)0;
    if (ph.kind == 1 && ph.beam) {
      // separable beam: amp * exp(-(x-cx)^2/w^2) * exp(-(y-cy)^2/w^2); centres from the host
      const R dx = (R)(ph.x[i] - sw.bc1x), dy = (R)(ph.x[j] - sw.bc1y), iw = (R)ph.beam_inv_w2;
      b1 = (R)ph.beam_amp * rexp(-dx * dx * iw) * rexp(-dy * dy * iw);
      if (two) {
        const R ex = (R)(ph.x[i] - sw.bc2x), ey = (R)(ph.x[j] - sw.bc2y);
        b2 = (R)ph.beam_amp * rexp(-ex * ex * iw) * rexp(-ey * ey * iw);
      }
    }
    if (ph.ltab) {
      // dynamic potential without z terms: this line's values at t1, t2
      const R* lt = (const R*)ph.ltab;
      b1 += lt[g];
      if (two) b2 += lt[(long long)N * N + g];
    }
    tb.c1[threadIdx.x] = base + b1;
    tb.c2[threadIdx.x] = base + b2;
    tb.c12[threadIdx.x] = pre ? ((base + b1) + (base + b2)) * h : (base + b1) + (base + b2);
  }
}

template <int N, typename R>
__device__ __forceinline__ void x_tables(const Phys& ph, int j, int k0, FastTables<R>& tb) {
  constexpr int L = FastCfg<N, R>::L, T = FastCfg<N, R>::T;
  for (int q = threadIdx.x; q < N; q += T) {
    tb.kx[q] = ph.kin[q];
    tb.kx2[q] = ph.k[q] * ph.k[q];
  }
  if (threadIdx.x < L) {
    const int k = k0 + threadIdx.x;
    const double2 a = ph.kin[j], b = ph.kin[k];
    // the inverse transforms' 1/M rides on the kinetic factor (one multiply per
    // line instead of one per element in the z sweep that follows)
    const double2 f = ph.kind == 0 ? make_double2(a.x * b.x, 0.0) : cmul(a, b);
    tb.kyz[threadIdx.x] = make_double2(f.x * ph.inv_m, f.y * ph.inv_m);
    tb.kyz2[threadIdx.x] = ph.k[j] * ph.k[j] + ph.k[k] * ph.k[k];
  }
}

// Kinetic factor of (i, line l) applied in FP64 (reference gpe/kernels.py:3-66);
// REAL / CUT are compile-time so the per-element code has no branches.
template <typename R, bool REAL, bool CUT>
__device__ __forceinline__ typename Cx<R>::T fast_kin(const Phys& ph, const FastTables<R>& tb,
                                                      typename Cx<R>::T v, int i, int l) {
  const double2 a = tb.kx[i], b = tb.kyz[l];
  const double vx = v.x, vy = v.y;
  typename Cx<R>::T out;
  if (!REAL) {
    const double f = a.x * b.x;
    out = mk((R)(vx * f), (R)(vy * f));
  } else {
    const double fx = a.x * b.x - a.y * b.y, fy = a.x * b.y + a.y * b.x;
    out = mk((R)(vx * fx - vy * fy), (R)(vx * fy + vy * fx));
  }
  if (CUT) {
    const bool drop = tb.kx2[i] + tb.kyz2[l] > ph.kcut2;
    out = drop ? mk((R)0, (R)0) : out;
  }
  return out;
}

// true when slot s of this thread exists in a layout with LANES lanes per line
template <int N, typename R, int LANES, int SLOTS>
__device__ __forceinline__ bool slot_ok(int s) {
  constexpr int L = FastCfg<N, R>::L, T = FastCfg<N, R>::T;
  return !(SLOTS * T > L * LANES) || (int)threadIdx.x + s * T < L * LANES;
}

template <int N, int AX, typename R, int LANES, int VALS, int SLOTS, int EPT, bool REAL, bool CUT>
__device__ __forceinline__ void kin_all(typename Cx<R>::T (&v)[EPT], const Phys& ph, const FastTables<R>& tb) {
  constexpr int L = FastCfg<N, R>::L, T = FastCfg<N, R>::T;
#pragma unroll
  for (int s = 0; s < SLOTS; ++s) {
    if (!slot_ok<N, R, LANES, SLOTS>(s)) break;
    int l, lane;
    slot<AX, L, T>(threadIdx.x + s * T, LANES, l, lane);
#pragma unroll
    for (int a = 0; a < VALS; ++a) v[s * VALS + a] = fast_kin<R, REAL, CUT>(ph, tb, v[s * VALS + a], lane + LANES * a, l);
  }
}

// One local half-step over all registers (layout LANES x VALS, element m = lane +
// LANES*a, Z tiles: m = z index), potential vz[m] + ctab[l] (+ arrays).  complex64:
// each element whose phase is within the short series' range (|phase| <= 1/8,
// first omitted terms below 8e-10 of the result) is rotated at once; the others
// are marked and, only when some lane of the warp has one, rotated in a second
// pass (full series up to pi/4, 1/2 in imaginary time; library sincosf/expm1f
// beyond).  No per-element phase array is kept across the two passes, which
// keeps the fused sweeps within their register budget.
// TWO: two consecutive real-time half-steps at one point as one rotation by
// (2 vz[m] + ctab[l] + 2 beta |psi|^2) dt/2 with ctab = c1 + c2; exact because
// the first rotation leaves |psi| unchanged.  The tables come prescaled (vz[m]
// by dt, ctab by dt/2, see z_tables) and callers pass beta as 2 beta dt/2.
template <int N, int AX, typename R, int LANES, int VALS, int SLOTS, int EPT, bool REAL, bool ARR,
          bool TWO = false>
__device__ __forceinline__ void half_all(typename Cx<R>::T (&v)[EPT], const FastTile<N, AX, R>& tl,
                                         const Phys& ph, const FastTables<R>& tb, const R* ctab,
                                         R beta, R h) {
  constexpr int L = FastCfg<N, R>::L, T = FastCfg<N, R>::T;
  static_assert(SLOTS * VALS <= 64, "pending mask");
  // complex64: elements whose phase exceeds the short series' range
  using Mask = typename std::conditional<(SLOTS * VALS <= 32), unsigned, unsigned long long>::type;
  Mask pend = 0;
#pragma unroll
  for (int s = 0; s < SLOTS; ++s) {
    if (!slot_ok<N, R, LANES, SLOTS>(s)) break;
    int l, lane;
    slot<AX, L, T>(threadIdx.x + s * T, LANES, l, lane);
    const long long row = tl.base + (long long)l * tl.lstride;
    const R c = ctab[l];
#pragma unroll
    for (int a = 0; a < VALS; ++a) {
      const int e = s * VALS + a, m = lane + LANES * a;
      R V = tb.vz[m] + c;
      R g = (R)0;
      if (ARR) {
        V += ph.vre ? ((const R*)ph.vre)[row + m] : (R)0;
        g = ph.vim ? ((const R*)ph.vim)[row + m] * h : (R)0;
      }
      const typename Cx<R>::T x = v[e];
      const R phs = TWO ? fma(beta, x.x * x.x + x.y * x.y, V) : (V + beta * (x.x * x.x + x.y * x.y)) * h;
      if (sizeof(R) == 8) {
        if (!REAL) {
          const double f = exp(-(double)phs);
          v[e] = mk((R)(x.x * f), (R)(x.y * f));
        } else {
          double sd, cd;
          sincos((double)phs, &sd, &cd);
          if (ARR) { const double am = exp((double)g); sd *= am; cd *= am; }
          v[e] = mk((R)(x.x * cd + x.y * sd), (R)(x.y * cd - x.x * sd));
        }
      } else if (fabs(phs) <= (R)0.125) {
        if (!REAL) {
          const float em = expm1_tiny((float)-phs);
          v[e] = mk(fma(x.x, (R)em, x.x), fma(x.y, (R)em, x.y));
        } else {
          float sn, cm1;
          sin_cosm1_tiny((float)phs, sn, cm1);
          if (ARR) { const float am = expm1f((float)g); cm1 = am + cm1 + am * cm1; sn = sn + sn * am; }
          v[e] = mk(fma(x.x, (R)cm1, fma(x.y, (R)sn, x.x)), fma(x.y, (R)cm1, fma(-x.x, (R)sn, x.y)));
        }
      } else {
        pend |= (Mask)1 << e;
      }
    }
  }
  if (sizeof(R) == 8 || !__any_sync(0xffffffffu, pend != 0)) return;
  // second pass over the elements left unrotated: full series up to pi/4 (1/2 in
  // imaginary time), library functions beyond
#pragma unroll
  for (int s = 0; s < SLOTS; ++s) {
    if (!slot_ok<N, R, LANES, SLOTS>(s)) break;
    int l, lane;
    slot<AX, L, T>(threadIdx.x + s * T, LANES, l, lane);
    const long long row = tl.base + (long long)l * tl.lstride;
    const R c = ctab[l];
#pragma unroll
    for (int a = 0; a < VALS; ++a) {
      const int e = s * VALS + a, m = lane + LANES * a;
      if (!((pend >> e) & 1)) continue;
      R V = tb.vz[m] + c;
      R g = (R)0;
      if (ARR) {
        V += ph.vre ? ((const R*)ph.vre)[row + m] : (R)0;
        g = ph.vim ? ((const R*)ph.vim)[row + m] * h : (R)0;
      }
      const typename Cx<R>::T x = v[e];
      const float p = (float)(TWO ? fma(beta, x.x * x.x + x.y * x.y, V) : (V + beta * (x.x * x.x + x.y * x.y)) * h);
      if (!REAL) {
        const float em = fabsf(p) <= 0.5f ? expm1_series(-p) : expm1f(-p);
        v[e] = mk(fma(x.x, (R)em, x.x), fma(x.y, (R)em, x.y));
      } else {
        float sn, cm1;
        if (fabsf(p) <= 0.78539816f) {
          sin_cosm1_series(p, sn, cm1);
        } else {
          float sh, ch;
          sincosf(0.5f * p, &sh, &ch);
          cm1 = -2.0f * sh * sh; sn = 2.0f * sh * ch;
        }
        if (ARR) { const float am = expm1f((float)g); cm1 = am + cm1 + am * cm1; sn = sn + sn * am; }
        v[e] = mk(fma(x.x, (R)cm1, fma(x.y, (R)sn, x.x)), fma(x.y, (R)cm1, fma(-x.x, (R)sn, x.y)));
      }
    }
  }
}

template <int N, int AX, typename R, int LANES, int VALS, int SLOTS, int EPT>
__device__ __forceinline__ void half_dispatch(typename Cx<R>::T (&v)[EPT], const FastTile<N, AX, R>& tl,
                                              const Phys& ph, const FastTables<R>& tb, const R* ctab) {
  const R beta = (R)ph.beta, h = (R)(ph.dt * 0.5);
  const bool arr = ph.vre != nullptr || ph.vim != nullptr;
  if (ph.kind == 1) {
    if (arr) half_all<N, AX, R, LANES, VALS, SLOTS, EPT, true, true>(v, tl, ph, tb, ctab, beta, h);
    else half_all<N, AX, R, LANES, VALS, SLOTS, EPT, true, false>(v, tl, ph, tb, ctab, beta, h);
  } else {
    if (arr) half_all<N, AX, R, LANES, VALS, SLOTS, EPT, false, true>(v, tl, ph, tb, ctab, beta, h);
    else half_all<N, AX, R, LANES, VALS, SLOTS, EPT, false, false>(v, tl, ph, tb, ctab, beta, h);
  }
}

// Diagnostic real-space sums of psi at time cx.t1 on the registers (layout LANES
// x VALS, element m = lane + LANES*a of line l), the terms of the reference's
// get_N and of E_pot, E_int (gpe/helper.py:81-93, 123-140): |psi|^2, V |psi|^2,
// |psi|^4 with the potential of the generic sweeps; a thread's values summed in
// plain FP64, the thread sums added with compensation.
template <int N, int AX, typename R, int LANES, int VALS, int SLOTS, int EPT>
__device__ __forceinline__ void diag_real_all(const typename Cx<R>::T (&v)[EPT], const FastTile<N, AX, R>& tl,
                                              const Phys& ph, const FastTables<R>& tb, PwCtx<R>& cx) {
  constexpr int L = FastCfg<N, R>::L, T = FastCfg<N, R>::T;
#pragma unroll
  for (int s = 0; s < SLOTS; ++s) {
    if (!slot_ok<N, R, LANES, SLOTS>(s)) break;
    int l, lane;
    slot<AX, L, T>(threadIdx.x + s * T, LANES, l, lane);
    double n0 = 0.0, n1 = 0.0, n2 = 0.0;
#pragma unroll
    for (int a = 0; a < VALS; ++a) {
      const int m = lane + LANES * a;
      int i, j, k;
      tl.coords(l, m, i, j, k);
      const typename Cx<R>::T x = v[s * VALS + a];
      const double rho = (double)x.x * x.x + (double)x.y * x.y;
      // with a line program the potential comes from the z-sweep tables (static
      // axes and line terms at t1), plus the static array
      const double V = ph.ltab ? (double)(tb.vz[m] + tb.c1[l] + (ph.vre ? ((const R*)ph.vre)[tl.gidx(l, m)] : (R)0))
                                : (double)potential<R>(ph, N, i, j, k, tl.gidx(l, m), cx.t1, cx.b1x, cx.b1y);
      n0 += rho;
      n1 = fma(V, rho, n1);
      n2 = fma(rho, rho, n2);
    }
    cx.acc[0].add(n0);
    cx.acc[1].add(n1);
    cx.acc[2].add(n2);
  }
}

// Diagnostic k-space sums of the transformed state (layout LANES x VALS after
// the x transform, frequency index m = lane + LANES*a): sum k^2 |psi_k|^2 (the
// reference's get_E) and, when cx.hist is set, the shell histogram of |psi_k|^2
// (gpe/nk_extraction.py:5-21); k^2 and the shell rule as in the generic sweeps.
template <int N, int AX, typename R, int LANES, int VALS, int SLOTS, int EPT>
__device__ __forceinline__ void diag_k_all(const typename Cx<R>::T (&v)[EPT], const FastTile<N, AX, R>& tl,
                                           const Phys& ph, PwCtx<R>& cx) {
  constexpr int L = FastCfg<N, R>::L, T = FastCfg<N, R>::T;
#pragma unroll
  for (int s = 0; s < SLOTS; ++s) {
    if (!slot_ok<N, R, LANES, SLOTS>(s)) break;
    int l, lane;
    slot<AX, L, T>(threadIdx.x + s * T, LANES, l, lane);
    double e = 0.0;
#pragma unroll
    for (int a = 0; a < VALS; ++a) {
      const int m = lane + LANES * a;
      int i, j, k;
      tl.coords(l, m, i, j, k);
      const typename Cx<R>::T x = v[s * VALS + a];
      const double kk = kk_ref(ph.k[i], ph.k[j], ph.k[k]);
      const double w = (double)x.x * x.x + (double)x.y * x.y;
      e = fma(kk, w, e);
      if (cx.hist) {
        int sh = (int)floor(sqrt(kk) / cx.shell_w + 0.5);
        sh = min(sh, cx.nbins - 1);
        atomicAdd(cx.hist + sh, w);
      }
    }
    cx.acc[3].add(e);
  }
}

// Pointwise stages of the fast modes on registers in layout (LANES lanes, VALS values).
template <int N, int AX, typename R, int MODE, int STAGE, int LANES, int VALS, int SLOTS, int EPT>
__device__ __forceinline__ void fast_pointwise(typename Cx<R>::T (&v)[EPT], const FastTile<N, AX, R>& tl,
                                               const Phys& ph, const FastTables<R>& tb, const FastOps& op,
                                               PwCtx<R>& cx) {
  if (MODE == FM_XKIN) {
    if (ph.kind == 1) {
      if (ph.kcut) kin_all<N, AX, R, LANES, VALS, SLOTS, EPT, true, true>(v, ph, tb);
      else kin_all<N, AX, R, LANES, VALS, SLOTS, EPT, true, false>(v, ph, tb);
    } else {
      kin_all<N, AX, R, LANES, VALS, SLOTS, EPT, false, false>(v, ph, tb);
    }
    return;
  }
  if (MODE == FM_Z1) {
    if (op.scale) {
      if (sizeof(R) == 8) {
#pragma unroll
        for (int e = 0; e < EPT; ++e) { v[e].x = (R)((double)v[e].x / cx.sc_div); v[e].y = (R)((double)v[e].y / cx.sc_div); }
      } else {
        scale_all(v, cx.sc_mul);
      }
    }
    half_dispatch<N, AX, R, LANES, VALS, SLOTS, EPT>(v, tl, ph, tb, tb.c1);
    return;
  }
  // (1/M was applied with the kinetic factor in the x sweep)
  if (MODE == FM_Z21 && ph.kind == 1 && ph.vre == nullptr && ph.vim == nullptr) {
    // real time, potential from tables: the two half-steps as one rotation
    const R h = (R)(ph.dt * 0.5);
    half_all<N, AX, R, LANES, VALS, SLOTS, EPT, true, false, true>(v, tl, ph, tb, tb.c12, (R)(2.0 * ph.beta) * h, h);
    return;
  }
  half_dispatch<N, AX, R, LANES, VALS, SLOTS, EPT>(v, tl, ph, tb, tb.c1);
  if (MODE == FM_Z21) half_dispatch<N, AX, R, LANES, VALS, SLOTS, EPT>(v, tl, ph, tb, tb.c2);
  if (MODE == FM_Z2 && op.norm) {
    // a thread's few values summed in plain FP64 (fixed order), the thread sums
    // then combined with compensation across the block and the grid
#pragma unroll
    for (int s = 0; s < SLOTS; ++s) {
      if (!slot_ok<N, R, LANES, SLOTS>(s)) break;
      double sum = 0.0;
#pragma unroll
      for (int a = 0; a < VALS; ++a) {
        const typename Cx<R>::T x = v[s * VALS + a];
        sum = fma((double)x.x, (double)x.x, fma((double)x.y, (double)x.y, sum));
      }
      cx.acc[0].add(sum);
    }
  }
}

// Load the tile into registers in layout (N1 lanes, N2 values); CG: through L2
// only (data another block wrote during the same launch).
template <int N, int AX, typename R, int S1, bool CG, int EPT>
__device__ __forceinline__ void fast_load(typename Cx<R>::T (&v)[EPT], const FastTile<N, AX, R>& tl,
                                          const typename Cx<R>::T* __restrict__ src, bool conj) {
  constexpr int L = FastCfg<N, R>::L, T = FastCfg<N, R>::T;
  constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
#pragma unroll
  for (int s = 0; s < S1; ++s) {
    if (!slot_ok<N, R, N1, S1>(s)) break;
    int l, lane;
    slot<AX, L, T>(threadIdx.x + s * T, N1, l, lane);
#pragma unroll
    for (int b = 0; b < N2; ++b) {
      const typename Cx<R>::T x = CG ? __ldcg(src + tl.gidx(l, lane + N1 * b)) : src[tl.gidx(l, lane + N1 * b)];
      v[s * N2 + b] = conj ? conj_<R>(x) : x;
    }
  }
}

template <int N, int AX, typename R, int LANES, int VALS, int SLOTS, int EPT>
__device__ __forceinline__ void fast_store(const typename Cx<R>::T (&v)[EPT], const FastTile<N, AX, R>& tl,
                                           typename Cx<R>::T* __restrict__ dst) {
  constexpr int L = FastCfg<N, R>::L, T = FastCfg<N, R>::T;
#pragma unroll
  for (int s = 0; s < SLOTS; ++s) {
    if (!slot_ok<N, R, LANES, SLOTS>(s)) break;
    int l, lane;
    slot<AX, L, T>(threadIdx.x + s * T, LANES, l, lane);
#pragma unroll
    for (int a = 0; a < VALS; ++a) dst[tl.gidx(l, lane + LANES * a)] = v[s * VALS + a];
  }
}

// Prefetch the lines of tile `tn` into L2 (128-byte lines; z tiles are one
// contiguous block, y/x tiles N rows of L elements).
template <int N, int AX, typename R>
__device__ __forceinline__ void fast_prefetch_l2(const FastTile<N, AX, R>& tn, const void* src) {
  using C = typename Cx<R>::T;
  constexpr int L = FastCfg<N, R>::L, T = FastCfg<N, R>::T;
  const C* base = (const C*)src + tn.base;
  if (AX == FZ) {
    constexpr int LINES = L * N * (int)sizeof(C) / 128;
    for (int q = threadIdx.x; q < LINES; q += T)
      asm volatile("prefetch.global.L2 [%0];" ::"l"(base + q * (128 / (int)sizeof(C))));
  } else {
    for (int m = threadIdx.x; m < N; m += T)
      asm volatile("prefetch.global.L2 [%0];" ::"l"(base + (long long)m * tn.nstride));
  }
}

// The sweep kernel of one mode.  Register layout before FFT #1: S1 slots of
// (N1 lanes, N2 values); after FFT #1: S2 slots of (N2 lanes, N1 values) =
// input layout of FFT #2 with (A, B) = (N2, N1); after FFT #2 the layout is
// back to (N1 lanes, N2 values).
//   FM_PLAIN  FFT (inverse if op.inv1; times 1/M if op.invm)       y sweeps, fftn/ifftn
//   FM_Z1     [scale] half(t1), forward                             first z sweep of a step
//   FM_Z2     inverse, half(t1) [norm partials]                     last z sweep of a step
//   FM_Z21    inverse, half(t1), half(t2), forward                  last z of a step + first z of the next
//   FM_XKIN   forward, kinetic x 1/M, inverse                       x sweep (carries the step's 1/M)
//   FM_DIAGR  real-space sums (N, E_pot, E_int), forward            diagnostic z sweep (to the work buffer)
//   FM_DIAGK  forward, k-space sums (E_kin [, shells]), no store     diagnostic x sweep
template <int N, int AX, typename R, int MODE, bool CG = false>
__device__ __forceinline__ void fast_body(const Phys& ph, const Sweep& sw, const FastOps& op, int tile,
                                          int ntiles) {
  using C = typename Cx<R>::T;
  constexpr int L = FastCfg<N, R>::L;
  constexpr int T = FastCfg<N, R>::T;
  constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
  constexpr int EPT = FastCfg<N, R>::V;   // registers (complex) per thread
  constexpr int S1 = FastCfg<N, R>::Q1;   // slots in layout (N1 lanes, N2 values)
  constexpr int S2 = FastCfg<N, R>::Q2;   // slots in layout (N2 lanes, N1 values)
  constexpr bool ZM = MODE == FM_Z1 || MODE == FM_Z2 || MODE == FM_Z21;
  // layout between the transforms: (N2 lanes, N1 values) after a two-phase
  // transform, (N1, N2) again after the three-phase one
  constexpr bool THREE = FastCfg<N, R>::THREE;
  constexpr int LM = THREE ? N1 : N2, VM = THREE ? N2 : N1, SM = THREE ? S1 : S2;
  using TW = typename TwE<R>::T;
  griddep_launch_dependents();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* ex = (C*)smem_raw + 2 * N;   // after the twiddle table (N entries of 16 bytes)
  Acc* red = (Acc*)(ex + fast_exchange_elems<N, R>());
  unsigned char* tail = (unsigned char*)(red + 32 * 4);
  FastTables<R> tb;
  tb.kx = (double2*)tail;
  tb.kyz = tb.kx + N;
  tb.kx2 = (double*)(tb.kyz + L);
  tb.kyz2 = tb.kx2 + N;
  tb.vz = (R*)(tb.kyz2 + L);
  tb.c1 = tb.vz + N;
  tb.c2 = tb.c1 + L;
  tb.c12 = tb.c2 + L;
  // 2-D twiddle tables: t1 for the split (N1 lanes, N2 values), t2 for (N2, N1);
  // complex64 entries pack hi and lo
  TW* t1 = (TW*)smem_raw;
  TW* t2 = (N1 == N2) ? t1 : (TW*)(tail + fast_tables_bytes<N, R>());
  const FastTile<N, AX, R> tl(tile);
  // shared-memory tables: plan constants only (twiddles, potential and kinetic tables)
  auto prologue = [&]() {
    const C* gh = (const C*)sw.tw;
    const C* gl = (const C*)sw.tw_lo;
    auto entry = [&](int e) -> TW {
      if constexpr (sizeof(R) == 4) return make_float4(gh[e].x, gh[e].y, gl[e].x, gl[e].y);
      else return gh[e];
    };
    for (int q = threadIdx.x; q < N; q += T) {
      const int k2 = q / N1, n1 = q % N1;   // t1[k2*N1 + n1] = W^(n1*k2), n1*k2 < N
      t1[q] = entry(n1 * k2);
      if (THREE) {
        // second-phase table of the three-phase transform: t2[k1*8 + p1] = W_64^(p1*k1)
        if (q < 64) t2[q] = entry(8 * ((q % 8) * (q / 8)));
      } else if (N1 != N2) {
        const int k2b = q / N2, n2 = q % N2;  // t2[k1*N2 + n2] = W^(n2*k1)
        t2[q] = entry(n2 * k2b);
      }
    }
    if (ZM || (MODE == FM_DIAGR && ph.ltab))
      z_tables<N, R>(ph, sw, tl.a0, tb, MODE == FM_Z21,
                     MODE == FM_Z21 && ph.kind == 1 && ph.vre == nullptr && ph.vim == nullptr);
    if (MODE == FM_XKIN) x_tables<N, R>(ph, tl.a0, tl.b0, tb);
    // diagnostic x sweep: the shell histogram takes the tables region
    if (MODE == FM_DIAGK && sw.hist)
      for (int b = threadIdx.x; b < sw.nbins; b += T) ((double*)tail)[b] = 0.0;
  };
  // psi and the renormalisation scale come from the previous sweep: read them
  // after the grid-dependency wait; the tile's loads are issued first and are in
  // flight while the tables are built (measured faster than building the tables
  // before the wait, where only the first wave would overlap them)
  griddep_wait();
  PwCtx<R> cx;
  cx.sc_div = 1.0;
  cx.sc_mul = (R)1;
  if (MODE == FM_Z1 && op.scale) {
    cx.sc_div = __ldcg(sw.scale);
    cx.sc_mul = (R)__ldcg(sw.scale + 1);
  }
  if (MODE == FM_DIAGR) {
    cx.t1 = sw.t1;
    cx.b1x = sw.bc1x;
    cx.b1y = sw.bc1y;
  }
  if (MODE == FM_DIAGK) {
    cx.hist = sw.hist ? (double*)tail : nullptr;
    cx.nbins = sw.nbins;
    cx.shell_w = sw.shell_w;
  }

  C v[EPT];
  fast_load<N, AX, R, S1, CG>(v, tl, (const C*)sw.src, MODE == FM_Z2 || MODE == FM_Z21 || (MODE == FM_PLAIN && op.inv1));
  // Bring the tile of the next wave's block on this SM into L2 while this one
  // computes: one wave ahead (tile + resident blocks), measured 51.2 -> 46.4 us
  // for the y sweep at 256^3 (two waves ahead was slower).
  if (!CG && op.pf > 0 && tile + op.pf < ntiles) fast_prefetch_l2<N, AX, R>(FastTile<N, AX, R>(tile + op.pf), sw.src);
  prologue();
  __syncthreads();  // twiddles and tables visible
  if (MODE == FM_Z1) fast_pointwise<N, AX, R, MODE, 0, N1, N2, S1>(v, tl, ph, tb, op, cx);
  if (MODE == FM_DIAGR) diag_real_all<N, AX, R, N1, N2, S1>(v, tl, ph, tb, cx);
  // the first transform frees the exchange buffer only when a second one follows
  constexpr bool TWO_FFT = MODE == FM_Z21 || MODE == FM_XKIN;
  if constexpr (THREE) fft_3phase<N, AX, R, S1, EPT, TWO_FFT>(v, ex, t1, t2);
  else fft_2phase<N, N1, N2, AX, R, S1, S2, EPT, false, TWO_FFT>(v, ex, t1);
  if (MODE == FM_Z21 || MODE == FM_XKIN) {
    if (MODE == FM_Z21) conj_all(v);  // finish the inverse before the physics
    fast_pointwise<N, AX, R, MODE, 1, LM, VM, SM>(v, tl, ph, tb, op, cx);
    if (MODE == FM_XKIN) conj_all(v);  // start the inverse
    if constexpr (THREE) fft_3phase<N, AX, R, S1, EPT, false>(v, ex, t1, t2);
    else fft_2phase<N, N2, N1, AX, R, S2, S1, EPT, false, false>(v, ex, t2);
    if (MODE == FM_XKIN) conj_all(v);
    fast_store<N, AX, R, N1, N2, S1>(v, tl, (C*)sw.dst);
  } else {
    if (MODE == FM_Z2 || (MODE == FM_PLAIN && op.inv1)) conj_all(v);
    if (MODE == FM_Z2) fast_pointwise<N, AX, R, MODE, 2, LM, VM, SM>(v, tl, ph, tb, op, cx);
    if (MODE == FM_PLAIN && op.invm) scale_all(v, (R)ph.inv_m);
    if (MODE == FM_DIAGK) diag_k_all<N, AX, R, LM, VM, SM>(v, tl, ph, cx);
    else fast_store<N, AX, R, LM, VM, SM>(v, tl, (C*)sw.dst);
  }
  if (MODE == FM_Z2 && op.norm) {
    Acc a[1] = {cx.acc[0]};
    block_merge<1>(a, red);
    norm_finish_n(ph, sw, a[0], red, tile, ntiles);
  }
  if (MODE == FM_DIAGR || MODE == FM_DIAGK) {
    // per-tile partials in the generic sweeps' layout: [tile][N, E_pot, E_int, E_kin]
    Acc a[4] = {cx.acc[0], cx.acc[1], cx.acc[2], cx.acc[3]};
    block_merge<4>(a, red);
    if (threadIdx.x == 0)
      for (int q = 0; q < 4; ++q) sw.partial[(long long)tile * 4 + q] = a[q].value();
    if (MODE == FM_DIAGK && sw.hist) {
      __syncthreads();
      for (int b = threadIdx.x; b < sw.nbins; b += T) sw.hist[(long long)tile * sw.nbins + b] = cx.hist[b];
    }
  }
}

// Resident blocks per SM that the register allocation must allow, 0 = the
// compiler's choice.  Measured for complex64 at n = 128, 256: the plain FFT
// sweeps are memory-bound and want 1024 threads per SM (64 registers at
// T = 256); the fused modes keep 768 (80 registers) for their extra live state,
// except Z21 and XKIN at n = 256, which run 4 blocks of 64 registers (a few
// hundred bytes of spills in Z21): 4486 -> 4541 steps/s at 256^3, the gain
// being in the overlap of the programmatically launched sweeps.
// At n = 512 (three radix-8 phases, 16 values per thread, 512-thread blocks of
// about 98 KB of shared memory) two blocks per SM, 64 registers: 378 -> 415
// steps/s at 512^3 against the earlier 32 x 16 split (32 values per thread, one
// block of 128 registers per SM).
// The diagnostic z sweep (FP64 potential per point) keeps 512 threads per SM.
template <int N, typename R, int MODE> struct FastBounds {
  static constexpr int value = (sizeof(R) == 4 && (N == 128 || N == 256))
                                   ? (MODE == FM_PLAIN ? 1024 : MODE == FM_DIAGR ? 512
                                      : (N == 256 && (MODE == FM_Z21 || MODE == FM_XKIN)) ? 1024 : 768) /
                                         FastCfg<N, R>::T
                               : (sizeof(R) == 4 && N == 512)
                                   ? (MODE == FM_DIAGR ? 512 : 1024) / FastCfg<N, R>::T : 0;
};

template <int N, int AX, typename R, int MODE>
__global__ void __launch_bounds__(FastCfg<N, R>::T) k_fast(Phys ph, Sweep sw, FastOps op) {
  fast_body<N, AX, R, MODE>(ph, sw, op, blockIdx.x, gridDim.x);
}

template <int N, int AX, typename R, int MODE, int B>
__global__ void __launch_bounds__(FastCfg<N, R>::T, B) k_fast_occ(Phys ph, Sweep sw, FastOps op) {
  fast_body<N, AX, R, MODE>(ph, sw, op, blockIdx.x, gridDim.x);
}

// Batched launch: blockIdx.y selects the instance (structs staged in shared memory).
template <int N, int AX, typename R, int MODE>
__device__ __forceinline__ void fast_batch_body(const Phys* __restrict__ phs, const Sweep* __restrict__ sws,
                                                const FastOps& op) {
  __shared__ Phys ph;
  __shared__ Sweep sw;
  if (threadIdx.x == 0) {
    ph = phs[blockIdx.y];
    sw = sws[blockIdx.y];
  }
  __syncthreads();
  if (batch_frozen(sw.live)) return;
  fast_body<N, AX, R, MODE>(ph, sw, op, blockIdx.x, gridDim.x);
}

template <int N, int AX, typename R, int MODE>
__global__ void __launch_bounds__(FastCfg<N, R>::T) k_fast_batch(const Phys* __restrict__ phs,
                                                                const Sweep* __restrict__ sws, FastOps op) {
  fast_batch_body<N, AX, R, MODE>(phs, sws, op);
}

template <int N, int AX, typename R, int MODE, int B>
__global__ void __launch_bounds__(FastCfg<N, R>::T, B) k_fast_batch_occ(const Phys* __restrict__ phs,
                                                                       const Sweep* __restrict__ sws, FastOps op) {
  fast_batch_body<N, AX, R, MODE>(phs, sws, op);
}


// ---------------------------------------------------------------- plane-fused sweeps
// The y and z sweeps of a step never leave an x-plane: a y tile (16 z columns
// of one plane) needs the whole plane's z sweep, a z tile (16 z lines) the
// whole plane's y sweep, and nothing else.  One persistent launch runs up to
// three consecutive y/z sweeps (e.g. inverse y, fused z, forward y) as a task
// list: task = (plane, stage, tile), handed out by an atomic ticket in an order
// where every task's dependencies hold smaller tickets (windows of W planes,
// software-pipelined: stage s of window w runs in block w + s).  A task of
// stage s > 0 waits (bounded) until the plane's stage s-1 count reaches its
// tile count; blocks that hold smaller tickets are resident and never wait on
// larger ones, so the wait always ends.  Intermediate planes stay in L2: psi
// crosses HBM once in and once out per launch instead of once per sweep.
struct PlaneJob {
  FastOps op[3];    // per stage
  int nstage;       // 1..3
  int zstage;       // the z stage; the others are y sweeps
  int window;       // planes per scheduling window (divides N)
  unsigned* ctr;    // [0] task ticket, [1] blocks finished, [2 + 3p + s] tiles done of (plane p, stage s)
};

// bounded wait of a plane-fused task (iterations of ~64 ns sleeps, ~0.3 s)
constexpr int PLANE_WAIT_LIMIT = 1 << 22;

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

template <int N, typename R, int MZ>
__device__ __forceinline__ void plane_body(const Phys& ph, const Sweep& sw, const PlaneJob& job) {
  constexpr int L = FastCfg<N, R>::L;
  constexpr int TPP = N / L;   // tiles per plane and stage
  static_assert(N % L == 0, "plane tiles");
  const int ns = job.nstage, W = job.window;
  const int nw = N / W;   // windows
  const unsigned per_stage = (unsigned)W * TPP;
  const unsigned total = (unsigned)N * TPP * ns;
  unsigned* ticket = job.ctr;
  unsigned* finished = job.ctr + 1;
  unsigned* done = job.ctr + 2;
  // tickets are fetched one task ahead so the atomic's latency hides behind a
  // task (a held, not yet started task waits on nothing, so the order argument
  // above still holds)
  __shared__ unsigned s_task[2];
  if (threadIdx.x == 0) s_task[0] = atomicAdd(ticket, 1u);
  for (int k = 0;; k ^= 1) {
    __syncthreads();  // the previous task is done with shared memory; s_task[k] visible
    const unsigned t = s_task[k];
    if (t >= total) break;
    if (threadIdx.x == 0) s_task[k ^ 1] = atomicAdd(ticket, 1u);
    // pipelined order: block b = [stage 0 of window b, stage 1 of window b-1,
    // stage 2 of window b-2]; a task's producer is ~3 windows of tiles earlier
    int s = 0, w = 0;
    unsigned q = t;
    for (int b = 0;; ++b) {
      const int s_lo = b - (nw - 1) > 0 ? b - (nw - 1) : 0, s_hi = b < ns - 1 ? b : ns - 1;
      const unsigned size = (unsigned)(s_hi - s_lo + 1) * per_stage;
      if (q < size) { s = s_lo + (int)(q / per_stage); w = b - s; q %= per_stage; break; }
      q -= size;
    }
    const int p = w * W + (int)(q / TPP), j = (int)(q % TPP);
    if (s > 0) {
      if (threadIdx.x == 0) {
        const unsigned* c = done + 3 * p + (s - 1);
        int it = 0;
        while (ld_acquire_u32(c) < (unsigned)TPP) {
          // after one timeout every later wait gives up at once
          if (++it > PLANE_WAIT_LIMIT || (*(volatile int*)sw.status & ST_TIMEOUT)) {
            atomicOr(sw.status, ST_TIMEOUT);
            break;
          }
          __nanosleep(64);
        }
      }
      __syncthreads();
    }
    const int tile = p * TPP + j;
    const FastOps op = s == 0 ? job.op[0] : (s == 1 ? job.op[1] : job.op[2]);
    if (s == job.zstage) fast_body<N, FZ, R, MZ, true>(ph, sw, op, tile, N * TPP);
    else fast_body<N, FY, R, FM_PLAIN, true>(ph, sw, op, tile, N * TPP);
    // release the tile: the barrier orders every thread's stores before thread
    // 0's gpu-scope fence, which makes them visible before the count
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(done + 3 * p + s, 1u);
    }
  }
  // the last block to finish resets the counters for the next launch (every
  // other block has taken its final ticket by then)
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(finished, 1u) == gridDim.x - 1) {
      for (int i = 0; i < 3 * N; ++i) done[i] = 0u;
      *ticket = 0u;
      __threadfence();
      *finished = 0u;
    }
  }
}

template <int N, typename R, int MZ>
__global__ void __launch_bounds__(FastCfg<N, R>::T, 768 / FastCfg<N, R>::T) k_plane(Phys ph, Sweep sw,
                                                                                    PlaneJob job) {
  plane_body<N, R, MZ>(ph, sw, job);
}

}  // namespace gpe
