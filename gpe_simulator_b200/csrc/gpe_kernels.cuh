// gpe_kernels.cuh -- fused split-step sweeps over psi (sm_100a).
//
// A Strang step is a sequence of sweeps; each sweep reads a tile of lines of
// psi from HBM into shared memory, applies pointwise work (renormalisation,
// local half-steps, 1/M, kinetic phase), runs the FFT passes along one axis
// and writes the tile back.  Pointwise work is attached to three points of a
// sweep: PRE (on the loaded values, before FFT #1), MID (between FFT #1 and
// FFT #2, on the tile in shared memory) and POST (on the values being stored).
// A pointwise stage applies, in this order: conjugate-in, pending scale,
// 1/M, half-step at t1, half-step at t2, kinetic factor, conjugate-out, norm
// accumulation.
#pragma once
#include "gpe_fft.cuh"
#include <math.h>

namespace gpe {

enum : unsigned {
  PW_CONJ_FIRST = 1u, PW_SCALE = 2u, PW_INVM = 4u, PW_HALF1 = 8u, PW_HALF2 = 16u,
  PW_KIN = 32u, PW_CONJ_LAST = 64u, PW_NORM = 128u, PW_DIAG_R = 256u, PW_DIAG_K = 512u,
  PW_LZ_X = 1024u, PW_LZ_Y = 2048u
};

enum Axis : int { AX_Z = 0, AX_Y = 1, AX_X = 2 };

// Internal opcodes of the line programs the host derives from a dynamic
// potential (beyond the public ones of gpe_ssf.h): square of the top of the
// stack, and push of slot k (OP_SLOT0 + k).
constexpr int OP_SQR = 40;
constexpr int OP_SLOT0 = 64;
#define GPE_LINE_SLOTS 8

// status bits
enum : int { ST_NONFINITE = 1, ST_TIMEOUT = 2, ST_LAYOUT = 4 };  // ST_LAYOUT: a sweep refused its shared-memory layout

struct Phys {
  int kind;              // 0 imaginary, 1 real
  double beta, dt, ckin;
  double inv_m, dx3;
  const double* x;       // axis coordinates [n]
  const double* k;       // axis wavenumbers [n]
  const double2* kin;    // per-axis kinetic factors [n]: exp(-i ckin k^2 dt) (real time) or (exp(-ckin k^2 dt), 0)
  const double* kth;     // per-axis kinetic phases [n]: ckin k^2 dt
  const void* vax;       // [3n] static axis potential, precision R
  const void* vre;       // [n^3] static real array, precision R (nullable)
  const void* vim;       // [n^3] static imaginary part (real time), precision R (nullable)
  const double* dyn;     // dynamic bytecode (nullable)
  int dyn_len;
  // register-resident sweeps: the dynamic potential when none of its terms depends
  // on z, per z-line (i n + j) at the two half-step times of the next z sweep:
  // [2][n*n] in precision R, filled by k_line_table right before that sweep
  const void* ltab;
  int beam;
  double beam_amp, beam_inv_w2, beam_radius, beam_omega, beam_t_ramp;
  int kcut;
  double kcut2;
  int local_fp64;        // complex64: evaluate the local half-step factor in FP64
  int exact_local;       // exact local sub-flows (FP64), not the reference's frozen density
};

struct Sweep {
  const void* src;
  void* dst;
  const void* tw;        // [n] forward twiddles W_n^j, precision of the sweep
  const void* tw_lo;     // [n] rounding residuals of tw (complex64), zeros (complex128)
  PassPlan pp;
  int lt;                // lines per tile
  int tiles_per_row;     // y/x tiles: ceil(n/lt)
  unsigned pre, mid, post;
  int fft1, fft2;        // run FFT #1 / #2
  double t1, t2;         // times of the half-steps PW_HALF1 / PW_HALF2 (t_mid of the step)
  double bc1x, bc1y;     // stirring-beam centre at t1 and t2 (FP64 angle, set by the host
  double bc2x, bc2y;     //   once per launch)
  double* partial;       // per-block partial sums (PW_NORM: 1 double; diag: several)
  unsigned* ticket;      // last-block ticket
  double* scale;         // [0] = sqrt(N) of the last renormalisation, [1] = 1/sqrt(N)
  int* status;
  int nbins;             // diag k-space: number of shells
  double shell_w;        // shell width
  double* hist;          // per-block shell histograms [gridDim][nbins]
  const int* live;       // batched imaginary-time instance: 0 = frozen (converged), its
                         // launches return at once; null: always advance
};

// A batched launch's instance is frozen: thread 0 reads the flag (written by an
// earlier launch on the stream) into shared memory; every thread returns alike.
__device__ __forceinline__ bool batch_frozen(const int* live) {
  __shared__ int s_live;
  if (threadIdx.x == 0) s_live = live ? __ldcg(live) : 1;
  __syncthreads();
  return s_live == 0;
}

// Values of a line program's slots (its time-dependent subexpressions, FP64,
// evaluated on the host) at the two half-step times of one z sweep.
struct LineSlots {
  double s1[GPE_LINE_SLOTS];
  double s2[GPE_LINE_SLOTS];
};

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}

// compensated accumulator
struct Acc {
  double s = 0.0, c = 0.0;
  __device__ __forceinline__ void add(double v) {
    double t, e;
    two_sum(s, v, t, e);
    s = t; c += e;
  }
  __device__ __forceinline__ void merge(const Acc& o) {
    double t, e;
    two_sum(s, o.s, t, e);
    s = t; c += o.c + e;
  }
  __device__ __forceinline__ double value() const { return s + c; }
};

__device__ __forceinline__ Acc warp_merge(Acc a) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    Acc b;
    b.s = __shfl_xor_sync(0xffffffffu, a.s, o);
    b.c = __shfl_xor_sync(0xffffffffu, a.c, o);
    a.merge(b);
  }
  return a;
}

// Deterministic block reduction of NV compensated accumulators; result valid in thread 0.
template <int NV>
__device__ void block_merge(Acc (&a)[NV], Acc* sh /* [32*NV] */) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int v = 0; v < NV; ++v) a[v] = warp_merge(a[v]);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int v = 0; v < NV; ++v) sh[w * NV + v] = a[v];
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      Acc b;
      if (lane < nw) b = sh[lane * NV + v];
      a[v] = warp_merge(b);
    }
  }
  __syncthreads();
}

// Potential-expression stack machine (FP64); `slots` serves the internal
// OP_SLOT0 + k pushes of line programs (null for the public bytecode).
static __device__ double eval_program(const double* prog, int len, double x, double y, double z, double t,
                                      const double* slots = nullptr) {
  double st[32];
  int sp = 0;
  for (int pc = 0; pc < len;) {
    const int op = (int)prog[pc++];
    switch (op) {
      case 1: st[sp++] = prog[pc++]; break;
      case 2: st[sp++] = x; break;
      case 3: st[sp++] = y; break;
      case 4: st[sp++] = z; break;
      case 5: st[sp++] = t; break;
      case 6: --sp; st[sp - 1] = st[sp - 1] + st[sp]; break;
      case 7: --sp; st[sp - 1] = st[sp - 1] - st[sp]; break;
      case 8: --sp; st[sp - 1] = st[sp - 1] * st[sp]; break;
      case 9: --sp; st[sp - 1] = st[sp - 1] / st[sp]; break;
      case 10: --sp; st[sp - 1] = pow(st[sp - 1], st[sp]); break;
      case 11: st[sp - 1] = -st[sp - 1]; break;
      case 13: st[sp - 1] = sin(st[sp - 1]); break;
      case 14: st[sp - 1] = cos(st[sp - 1]); break;
      case 15: st[sp - 1] = tan(st[sp - 1]); break;
      case 16: st[sp - 1] = exp(st[sp - 1]); break;
      case 17: st[sp - 1] = sqrt(st[sp - 1]); break;
      case 18: st[sp - 1] = tanh(st[sp - 1]); break;
      case 19: st[sp - 1] = fabs(st[sp - 1]); break;
      case 20: st[sp - 1] = log(st[sp - 1]); break;
      case OP_SQR: st[sp - 1] = st[sp - 1] * st[sp - 1]; break;
      default:
        if (slots && op >= OP_SLOT0 && op < OP_SLOT0 + GPE_LINE_SLOTS) st[sp++] = slots[op - OP_SLOT0];
        break;
    }
    if (sp < 1) sp = 1;
    if (sp > 31) sp = 31;
  }
  return st[0];
}

// The dynamic potential of every z-line (i n + j) at t1 (and t2 when `two`),
// FP64 evaluation of the line program stored in precision R: one thread per
// line and time.  Launched as a programmatic dependent of the sweep before it,
// it waits for that sweep (the z sweep that last read the table has finished by
// then) and lets the z sweep after it launch early.
template <typename R>
__global__ void __launch_bounds__(256) k_line_table(const double* __restrict__ prog, int len,
                                                    const double* __restrict__ x, int n, LineSlots sl,
                                                    R* __restrict__ tab, int two) {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const long long nn = (long long)n * n;
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (two ? 2 : 1) * nn) return;
  const int which = (int)(q / nn);
  const long long l = q - which * nn;
  tab[q] = (R)eval_program(prog, len, x[l / n], x[l % n], 0.0, 0.0, which ? sl.s2 : sl.s1);
}

// Beam centre for a time; angle accumulated in FP64.
__device__ __forceinline__ void rsincos(float a, float* s, float* c) { sincosf(a, s, c); }
__device__ __forceinline__ void rsincos(double a, double* s, double* c) { sincos(a, s, c); }
__device__ __forceinline__ float rexp(float a) { return expf(a); }
__device__ __forceinline__ double rexp(double a) { return exp(a); }

// Real potential at point (i,j,k) for time t (precision R).
template <typename R>
__device__ __forceinline__ R potential(const Phys& ph, int n, int i, int j, int k, long long idx,
                                       double t, double bcx, double bcy) {
  const R* vax = (const R*)ph.vax;
  R v = vax[i] + vax[n + j] + vax[2 * n + k];
  if (ph.vre) v += ((const R*)ph.vre)[idx];
  if (ph.kind == 1) {
    if (ph.beam) {
      const R dxb = (R)(ph.x[i] - bcx), dyb = (R)(ph.x[j] - bcy);
      v += (R)ph.beam_amp * rexp(-(dxb * dxb + dyb * dyb) * (R)ph.beam_inv_w2);
    }
    if (ph.dyn) v += (R)eval_program(ph.dyn, ph.dyn_len, ph.x[i], ph.x[j], ph.x[k], t);
  }
  return v;
}

// Local half-step at time t (reference gpe/make_kernel.py:14-45, 54-83, 93-119).
template <typename R>
__device__ __forceinline__ typename Cx<R>::T halfstep(const Phys& ph, typename Cx<R>::T v, int n, int i,
                                                      int j, int k, long long idx, double t, double bcx,
                                                      double bcy) {
  const R V = potential<R>(ph, n, i, j, k, idx, t, bcx, bcy);
  if (ph.exact_local) {
    // exact flows of the local subproblem over h = dt/2 (V held fixed):
    //   imaginary  d psi/dt = -(V + beta|psi|^2) psi:
    //              psi e^{-Vh} / sqrt(1 + 2 beta |psi|^2 s), s = (1 - e^{-2Vh}) / (2V)
    //   real       i d psi/dt = (V - i Gamma + beta|psi|^2) psi: |psi|^2 decays as e^{-2 Gamma t},
    //              phase V h + beta |psi|^2 tau, tau = (1 - e^{-2 Gamma h}) / (2 Gamma)
    const double vx = v.x, vy = v.y, h = ph.dt * 0.5, rho = vx * vx + vy * vy, Vd = (double)V;
    if (ph.kind == 0) {
      const double s = Vd == 0.0 ? h : -expm1(-2.0 * Vd * h) / (2.0 * Vd);
      const double f = exp(-Vd * h) / sqrt(1.0 + 2.0 * ph.beta * rho * s);
      return mk((R)(vx * f), (R)(vy * f));
    }
    const double g = ph.vim ? -(double)((const R*)ph.vim)[idx] : 0.0;   // Gamma
    const double tau = g == 0.0 ? h : -expm1(-2.0 * g * h) / (2.0 * g);
    double sd, cd;
    sincos(Vd * h + ph.beta * rho * tau, &sd, &cd);
    const double a = exp(-g * h);
    return mk((R)((vx * cd + vy * sd) * a), (R)((vy * cd - vx * sd) * a));
  }
  if (sizeof(R) == 4 && ph.local_fp64) {
    // complex64 data, local factor evaluated and applied in FP64
    const double vx = v.x, vy = v.y, hd = ph.dt * 0.5;
    const double phd = ((double)V + ph.beta * (vx * vx + vy * vy)) * hd;
    if (ph.kind == 0) {
      const double f = exp(-phd);
      return mk((R)(vx * f), (R)(vy * f));
    }
    double sd, cd;
    sincos(phd, &sd, &cd);
    if (ph.vim) {
      const double a = exp((double)((const R*)ph.vim)[idx] * hd);
      cd *= a; sd *= a;
    }
    return mk((R)(vx * cd + vy * sd), (R)(vy * cd - vx * sd));
  }
  const R h = (R)(ph.dt * 0.5);
  const R phase = (V + (R)ph.beta * (v.x * v.x + v.y * v.y)) * h;
  if (sizeof(R) == 4) {
    // complex64: v + v*(f - 1) with f - 1 from expm1 / half-angle sin-cos, so the
    // rounding of the factor scales with the (small) phase instead of with 1
    if (ph.kind == 0) {
      const R e = (R)expm1f((float)-phase);
      return mk(fma(v.x, e, v.x), fma(v.y, e, v.y));
    }
    float sh, ch;
    sincosf(0.5f * (float)phase, &sh, &ch);
    R cm1 = (R)(-2.0f * sh * sh), sn = (R)(2.0f * sh * ch);   // cos - 1, sin
    if (ph.vim) {
      const R am1 = (R)expm1f((float)(((const R*)ph.vim)[idx] * h));  // exp(-Gamma h) - 1
      cm1 = am1 + cm1 + am1 * cm1;
      sn = sn + sn * am1;
    }
    return mk(fma(v.x, cm1, fma(v.y, sn, v.x)), fma(v.y, cm1, fma(-v.x, sn, v.y)));
  }
  if (ph.kind == 0) {
    const R f = rexp(-phase);
    return mk(v.x * f, v.y * f);
  }
  R s, c;
  rsincos(phase, &s, &c);
  if (ph.vim) {
    const R a = rexp(((const R*)ph.vim)[idx] * h);
    c *= a; s *= a;
  }
  // v * (c - i s)
  return mk(v.x * c + v.y * s, v.y * c - v.x * s);
}

// Kinetic factor at wavenumber indices (i,j,k) applied in FP64
// (reference gpe/kernels.py:3-66).
template <typename R>
__device__ __forceinline__ typename Cx<R>::T kinetic(const Phys& ph, typename Cx<R>::T v, int n, int i,
                                                     int j, int k) {
  if (ph.kcut) {
    const double kk = ph.k[i] * ph.k[i] + ph.k[j] * ph.k[j] + ph.k[k] * ph.k[k];
    if (kk > ph.kcut2) return mk((R)0, (R)0);
  }
  if (sizeof(R) == 4 && ph.kind == 0) {
    // complex64 imaginary time: exponent summed in FP64, factor applied as v + v*(f - 1)
    // (the renormalisation absorbs modulus rounding).  Real time keeps the FP64 factor
    // below: the same per-mode factor every step makes any FP32 modulus rounding
    // accumulate as norm drift.
    const float th = (float)(ph.kth[i] + ph.kth[j] + ph.kth[k]);
    const R e = (R)expm1f(-th);
    return mk(fma(v.x, e, v.x), fma(v.y, e, v.y));
  }
  const double2 a = ph.kin[i], b = ph.kin[j], c = ph.kin[k];
  double2 f;
  if (ph.kind == 0) {
    f = make_double2(a.x * b.x * c.x, 0.0);
    return mk((R)((double)v.x * f.x), (R)((double)v.y * f.x));
  }
  f = cmul(cmul(a, b), c);
  const double vx = v.x, vy = v.y;
  return mk((R)(vx * f.x - vy * f.y), (R)(vx * f.y + vy * f.x));
}

// |k|^2 = kx^2 + ky^2 + kz^2 rounded as NumPy evaluates it (each product and sum
// rounded, left to right, no fused multiply-add), so shell indices at exact
// boundaries agree with the reference's nk_extraction.
__device__ __forceinline__ double kk_ref(double kx, double ky, double kz) {
  return __dadd_rn(__dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky)), __dmul_rn(kz, kz));
}

// Per-point pointwise stage.
template <typename R>
struct PwCtx {
  double t1, t2;
  double b1x, b1y, b2x, b2y;  // beam centres at t1, t2
  R sc_mul;                   // 1/sqrt(N) (float path)
  double sc_div;              // sqrt(N) (double path)
  Acc acc[4];                 // norm / diag accumulators
  double* hist;               // shared-memory shell histogram (PW_DIAG_K)
  int nbins;
  double shell_w;
};

template <typename R>
__device__ __forceinline__ typename Cx<R>::T pointwise(const Phys& ph, unsigned ops, typename Cx<R>::T v,
                                                       int n, int i, int j, int k, PwCtx<R>& cx) {
  const long long idx = ((long long)i * n + j) * n + k;
  if (ops & PW_CONJ_FIRST) v.y = -v.y;  // finishes an inverse transform
  if (ops & PW_SCALE) {
    if (sizeof(R) == 8) { v.x = (R)((double)v.x / cx.sc_div); v.y = (R)((double)v.y / cx.sc_div); }
    else { v.x *= cx.sc_mul; v.y *= cx.sc_mul; }
  }
  if (ops & PW_INVM) { v.x *= (R)ph.inv_m; v.y *= (R)ph.inv_m; }
  if (ops & PW_DIAG_R) {
    const double rho = (double)v.x * v.x + (double)v.y * v.y;
    const double V = (double)potential<R>(ph, n, i, j, k, idx, cx.t1, cx.b1x, cx.b1y);
    cx.acc[0].add(rho);
    cx.acc[1].add(V * rho);
    cx.acc[2].add(rho * rho);
  }
  if (ops & PW_HALF1) v = halfstep<R>(ph, v, n, i, j, k, idx, cx.t1, cx.b1x, cx.b1y);
  if (ops & PW_HALF2) v = halfstep<R>(ph, v, n, i, j, k, idx, cx.t2, cx.b2x, cx.b2y);
  if (ops & PW_KIN) v = kinetic<R>(ph, v, n, i, j, k);
  if (ops & PW_CONJ_LAST) v.y = -v.y;  // starts an inverse transform
  if (ops & PW_NORM) cx.acc[0].add((double)v.x * v.x + (double)v.y * v.y);
  if (ops & PW_DIAG_K) {
    // reference gpe/helper.py:116-121 and gpe/nk_extraction.py:5-13
    const double kk = kk_ref(ph.k[i], ph.k[j], ph.k[k]);
    const double w = (double)v.x * v.x + (double)v.y * v.y;
    cx.acc[3].add(kk * w);
    int sh = (int)floor(sqrt(kk) / cx.shell_w + 0.5);
    sh = min(sh, cx.nbins - 1);
    atomicAdd(cx.hist + sh, w);
  }
  // angular momentum terms (reference gpe/helper.py:143-156) on data transformed
  // along z and then x (LZ_X: y k_x |v|^2) or along z and then y (LZ_Y: x k_y |v|^2)
  if (ops & PW_LZ_X) cx.acc[3].add(ph.x[j] * ph.k[i] * ((double)v.x * v.x + (double)v.y * v.y));
  if (ops & PW_LZ_Y) cx.acc[3].add(ph.x[i] * ph.k[j] * ((double)v.x * v.x + (double)v.y * v.y));
  return v;
}

// ---------------------------------------------------------------- tile geometry
// z tiles: lt consecutive lines (line g = x*n + y), smem [l][pitch].
// y tiles: fixed x, z block of lt, smem [j][lt].   x tiles: fixed y, z block, smem [i][lt].
template <int AX>
struct Tile {
  int n, lt, pitch;
  long long base;     // global index of element (line 0, index 0)
  long long lstride;  // global stride between lines
  long long nstride;  // global stride along the transform axis
  int nlines;         // valid lines in this tile
  int a0, b0;         // tile origin: z: first line g; y: (x, z0); x: (y, z0)
  __device__ Tile(int n_, int lt_, int tpr, int tile) : n(n_), lt(lt_) {
    if (AX == AX_Z) {
      pitch = (n & 1) ? n : n + 1;
      a0 = tile * lt; b0 = 0;
      nlines = min(lt, n * n - a0);
      base = (long long)a0 * n; lstride = n; nstride = 1;
    } else {
      pitch = lt;
      const int row = tile / tpr, z0 = (tile % tpr) * lt;
      a0 = row; b0 = z0;
      nlines = min(lt, n - z0);
      lstride = 1;
      if (AX == AX_Y) { base = (long long)row * n * n + z0; nstride = n; }
      else { base = (long long)row * n + z0; nstride = (long long)n * n; }
    }
  }
  __device__ __forceinline__ int sidx(int l, int m) const {
    return AX == AX_Z ? l * pitch + m : m * lt + l;
  }
  __device__ __forceinline__ void coords(int l, int m, int& i, int& j, int& k) const {
    if (AX == AX_Z) { const int g = a0 + l; i = g / n; j = g - i * n; k = m; }
    else if (AX == AX_Y) { i = a0; j = m; k = b0 + l; }
    else { i = m; j = a0; k = b0 + l; }
  }
  __device__ __forceinline__ int sn() const { return AX == AX_Z ? 1 : lt; }
  __device__ __forceinline__ int sl() const { return AX == AX_Z ? pitch : 1; }
};

template <typename R>
__device__ void setup_ctx(const Phys& ph, const Sweep& sw, unsigned all_ops, PwCtx<R>& cx) {
  cx.t1 = sw.t1;
  cx.t2 = sw.t2;
  cx.b1x = sw.bc1x;
  cx.b1y = sw.bc1y;
  cx.b2x = sw.bc2x;
  cx.b2y = sw.bc2y;
  cx.sc_div = 1.0;
  cx.sc_mul = (R)1;
  if (all_ops & PW_SCALE) {
    cx.sc_div = __ldcg(sw.scale);
    cx.sc_mul = (R)__ldcg(sw.scale + 1);
  }
}

// Finish a norm reduction: the last block to arrive sums all partials in a
// fixed order and stores sqrt(N) and 1/sqrt(N).
// Partial `total` of tile `idx` of `count`; the block that finishes last sums the
// partials in index order (deterministic) and publishes the renormalisation scale.
static __device__ void norm_finish_n(const Phys& ph, const Sweep& sw, Acc total, Acc* sh, int idx, int count) {
  __shared__ bool last;
  if (threadIdx.x == 0) {
    sw.partial[idx] = total.value();
    __threadfence();
    const unsigned t = atomicAdd(sw.ticket, 1u);
    last = (t == (unsigned)count - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  Acc a[1];
  for (int b = threadIdx.x; b < count; b += blockDim.x) a[0].add(__ldcg(sw.partial + b));
  block_merge<1>(a, sh);
  if (threadIdx.x == 0) {
    const double N = a[0].value() * ph.dx3;
    if (!(N > 0.0) || !isfinite(N)) atomicOr(sw.status, ST_NONFINITE);
    const double s = sqrt(N);
    sw.scale[0] = s;
    sw.scale[1] = 1.0 / s;
    sw.scale[2] = N;
    *sw.ticket = 0u;
  }
}

static __device__ void norm_finish(const Phys& ph, const Sweep& sw, Acc total, Acc* sh) {
  norm_finish_n(ph, sw, total, sh, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------- the sweep kernel
template <typename R, int AX, int EPT, bool GEN>
__device__ __forceinline__ void sweep_body(const Phys& ph, const Sweep& sw) {
  using C = typename Cx<R>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = sw.pp.n;
  Tile<AX> tl(n, sw.lt, sw.tiles_per_row, blockIdx.x);
  C* tw = (C*)smem_raw;
  C* twl = tw + n;
  C* s = twl + n;
  Acc* red = (Acc*)(s + (AX == AX_Z ? sw.lt * tl.pitch : n * sw.lt));
  const bool need_tw = sw.fft1 || sw.fft2;
  if (need_tw)
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
      tw[q] = ((const C*)sw.tw)[q];
      twl[q] = ((const C*)sw.tw_lo)[q];
    }

  PwCtx<R> cx;
  setup_ctx<R>(ph, sw, sw.pre | sw.mid | sw.post, cx);
  cx.hist = (double*)(red + 32 * 4);
  cx.nbins = sw.nbins;
  cx.shell_w = sw.shell_w;
  if ((sw.pre | sw.mid | sw.post) & PW_DIAG_K)
    for (int b = threadIdx.x; b < sw.nbins; b += blockDim.x) cx.hist[b] = 0.0;

  // load + PRE
  const C* __restrict__ src = (const C*)sw.src;
  const int E = n * sw.lt;
  for (int e = threadIdx.x; e < E; e += blockDim.x) {
    int l, m;
    if (AX == AX_Z) { l = e / n; m = e - l * n; }
    else { m = e / sw.lt; l = e - m * sw.lt; }
    C v = mk((R)0, (R)0);
    if (l < tl.nlines) {
      v = src[tl.base + (long long)l * tl.lstride + (long long)m * tl.nstride];
      if (sw.pre) { int i, j, k; tl.coords(l, m, i, j, k); v = pointwise<R>(ph, sw.pre, v, n, i, j, k, cx); }
    }
    s[tl.sidx(l, m)] = v;
  }
  __syncthreads();
  if (sw.fft1) fft_lines<EPT, GEN>(s, tw, twl, sw.pp, sw.lt, tl.sn(), tl.sl());
  if (sw.mid) {
    for (int e = threadIdx.x; e < E; e += blockDim.x) {
      int l, m;
      if (AX == AX_Z) { l = e / n; m = e - l * n; }
      else { m = e / sw.lt; l = e - m * sw.lt; }
      if (l < tl.nlines) {
        int i, j, k; tl.coords(l, m, i, j, k);
        const int si = tl.sidx(l, m);
        s[si] = pointwise<R>(ph, sw.mid, s[si], n, i, j, k, cx);
      }
    }
    __syncthreads();
  }
  if (sw.fft2) fft_lines<EPT, GEN>(s, tw, twl, sw.pp, sw.lt, tl.sn(), tl.sl());

  // POST + store
  C* __restrict__ dst = (C*)sw.dst;
  const bool store = dst != nullptr;
  for (int e = threadIdx.x; e < E; e += blockDim.x) {
    int l, m;
    if (AX == AX_Z) { l = e / n; m = e - l * n; }
    else { m = e / sw.lt; l = e - m * sw.lt; }
    if (l < tl.nlines) {
      C v = s[tl.sidx(l, m)];
      int i, j, k; tl.coords(l, m, i, j, k);
      if (sw.post) v = pointwise<R>(ph, sw.post, v, n, i, j, k, cx);
      if (store) dst[tl.base + (long long)l * tl.lstride + (long long)m * tl.nstride] = v;
    }
  }
  const unsigned all = sw.pre | sw.mid | sw.post;
  if (all & PW_NORM) {
    Acc a[1] = {cx.acc[0]};
    block_merge<1>(a, red);
    norm_finish(ph, sw, a[0], red);
  }
  if (all & (PW_DIAG_R | PW_DIAG_K | PW_LZ_X | PW_LZ_Y)) {
    Acc a[4] = {cx.acc[0], cx.acc[1], cx.acc[2], cx.acc[3]};
    block_merge<4>(a, red);
    if (threadIdx.x == 0)
      for (int v = 0; v < 4; ++v) sw.partial[blockIdx.x * 4 + v] = a[v].value();
    if (all & PW_DIAG_K) {
      __syncthreads();
      for (int b = threadIdx.x; b < sw.nbins; b += blockDim.x)
        sw.hist[(long long)blockIdx.x * sw.nbins + b] = cx.hist[b];
    }
  }
}

// Single-plan launch (structs by value) and batched launch: blockIdx.y selects the
// instance whose structs are staged once into shared memory.
template <typename R, int AX, int EPT, bool GEN>
__global__ void __launch_bounds__(512, 1) k_sweep(Phys ph, Sweep sw) {
  sweep_body<R, AX, EPT, GEN>(ph, sw);
}

template <typename R, int AX, int EPT, bool GEN>
__global__ void __launch_bounds__(512, 1) k_sweep_batch(const Phys* __restrict__ phs,
                                                         const Sweep* __restrict__ sws) {
  __shared__ Phys ph;
  __shared__ Sweep sw;
  if (threadIdx.x == 0) {
    ph = phs[blockIdx.y];
    sw = sws[blockIdx.y];
  }
  __syncthreads();
  if (batch_frozen(sw.live)) return;
  sweep_body<R, AX, EPT, GEN>(ph, sw);
}

}  // namespace gpe
