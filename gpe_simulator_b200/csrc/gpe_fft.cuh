// gpe_fft.cuh -- shared-memory mixed-radix FFT building blocks (sm_100a).
//
// A tile of `nl` lines of length `n` lives in shared memory with element
// (line l, index i) at s[l*sl + i*sn].  Each Stockham pass of radix R turns
// butterfly (l, i), i < n/R, with p = product of the earlier radices:
//     k = i mod p;  v[m] = s[l, i + m*n/R] * W_{pR}^{m k};  V = DFT_R(v);
//     s[l, (i-k)*R + k + m*p] = V[m]
// which leaves the transform in natural order after the last pass.  A pass is
// in place: every thread first gathers all of its butterflies into registers,
// the block synchronises, then every thread scatters.  Butterflies are
// numbered line-fastest, so consecutive lanes touch consecutive lines; with an
// odd line pitch (z lines) or unit line stride (y/x lines) the shared-memory
// accesses are bank-conflict free.
//
// Only the forward transform (W = exp(-2 pi i/n)) is implemented; the inverse
// is conj(FFT(conj(x))), with the conjugations folded into the pointwise work
// before and after the passes.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <type_traits>

namespace gpe {

template <typename R> struct Cx;
template <> struct Cx<float>  { using T = float2; };
template <> struct Cx<double> { using T = double2; };

__device__ __forceinline__ float2  mk(float a, float b)   { return make_float2(a, b); }
__device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return mk(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return mk(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C, typename R> __device__ __forceinline__ C cscale(C a, R s) { return mk(a.x * s, a.y * s); }
template <typename C> __device__ __forceinline__ C cconj(C a) { return mk(a.x, -a.y); }
// multiply by -i
template <typename C> __device__ __forceinline__ C cmi(C a) { return mk(a.y, -a.x); }

// ---------------------------------------------------------------- constants
// Unit-circle constants of the small DFTs.  For complex64 every constant is
// carried as a float pair hi + lo (hi = the rounded value, lo = the rounding
// residual) and applied as fma(x, hi, x*lo): a single rounded float would have
// |c + i s| != 1 by up to 6e-8, and because every butterfly multiplies by the
// same constants that error would bias the norm of every transform (and, in
// imaginary time, shift the fixed point).  With the split, value and modulus
// are exact to ~1e-15 and only unbiased arithmetic rounding remains.
// complex128 uses the correctly rounded doubles.
template <typename R> struct K;
template <> struct K<double> {
  static constexpr double C8 = 0.9238795325112867, C8L = 0;   // cos pi/8
  static constexpr double S8 = 0.3826834323650898, S8L = 0;   // sin pi/8
  static constexpr double R2 = 0.7071067811865476, R2L = 0;   // sqrt(1/2)
  static constexpr double H3 = 0.8660254037844386, H3L = 0;   // sin 2pi/3
  static constexpr double C1 = 0.30901699437494745, C1L = 0;  // cos 2pi/5
  static constexpr double S1 = 0.9510565162951535, S1L = 0;   // sin 2pi/5
  static constexpr double C2 = -0.8090169943749475, C2L = 0;  // cos 4pi/5
  static constexpr double S2 = 0.5877852522924731, S2L = 0;   // sin 4pi/5
};
template <> struct K<float> {
  static constexpr float C8 = 0.9238795042037964f, C8L = 2.830748968563057e-08f;
  static constexpr float S8 = 0.3826834261417389f, S8L = 6.2233507236442165e-09f;
  static constexpr float R2 = 0.7071067690849304f, R2L = 1.2101617485882343e-08f;
  static constexpr float H3 = 0.8660253882408142f, H3L = 1.5543625053737742e-08f;
  static constexpr float C1 = 0.30901700258255005f, C1L = -8.207602597565256e-09f;
  static constexpr float S1 = 0.9510565400123596f, S1L = -2.3717205976936384e-08f;
  static constexpr float C2 = -0.80901700258255f, C2L = 8.207602597565256e-09f;
  static constexpr float S2 = 0.5877852439880371f, S2L = 8.304436249773062e-09f;
};

// x * (hi + lo)
__device__ __forceinline__ float kmul(float x, float hi, float lo) { return fmaf(x, hi, x * lo); }
__device__ __forceinline__ double kmul(double x, double hi, double) { return x * hi; }

// v * (c - i s) for split constants c = ch + cl, s = sh + sl
__device__ __forceinline__ float2 rot(float2 v, float ch, float cl, float sh, float sl) {
  return make_float2(fmaf(v.x, ch, fmaf(v.y, sh, v.x * cl + v.y * sl)),
                     fmaf(v.y, ch, fmaf(-v.x, sh, v.y * cl - v.x * sl)));
}
__device__ __forceinline__ double2 rot(double2 v, double ch, double, double sh, double) {
  return make_double2(v.x * ch + v.y * sh, v.y * ch - v.x * sh);
}

// v * w for a table twiddle w = hi + lo (lo only for complex64)
__device__ __forceinline__ float2 twmul(float2 v, float2 w, float2 l) {
  return make_float2(fmaf(v.x, w.x, fmaf(-v.y, w.y, v.x * l.x - v.y * l.y)),
                     fmaf(v.x, w.y, fmaf(v.y, w.x, v.x * l.y + v.y * l.x)));
}
__device__ __forceinline__ double2 twmul(double2 v, double2 w, double2) { return cmul(v, w); }

// twiddle-table entries of the register-resident sweeps: complex64 keeps the
// {hi, lo} pair of a twiddle in one 16-byte entry (one shared-memory load),
// complex128 the twiddle itself
template <typename R> struct TwE;
template <> struct TwE<float>  { using T = float4; };
template <> struct TwE<double> { using T = double2; };
__device__ __forceinline__ float2 tw_apply(float2 v, float4 w) {
  return twmul(v, make_float2(w.x, w.y), make_float2(w.z, w.w));
}
__device__ __forceinline__ double2 tw_apply(double2 v, double2 w) { return cmul(v, w); }

// v * W_16^q, W_16 = exp(-2 pi i / 16), q known at compile time after unrolling
template <typename C> __device__ __forceinline__ C mul_w16(C v, int q) {
  using R = decltype(v.x);
  using k = K<R>;
  q &= 15;
  if (q == 0) return v;
  if (q == 4) return cmi(v);
  if (q == 8) return mk(-v.x, -v.y);
  if (q == 12) return mk(-v.y, v.x);
  if ((q & 1) == 0) {
    // odd multiples of pi/4: sqrt(1/2) * (a + i b), a, b = +-1
    const R a = (q == 2 || q == 14) ? R(1) : R(-1);
    const R b = (q == 2 || q == 6) ? R(-1) : R(1);
    return mk(kmul(a * v.x - b * v.y, k::R2, k::R2L), kmul(a * v.y + b * v.x, k::R2, k::R2L));
  }
  // odd multiples of pi/8: v * (cos - i sin) of pi q / 8
  switch (q) {
    case 1:  return rot(v, k::C8, k::C8L, k::S8, k::S8L);
    case 3:  return rot(v, k::S8, k::S8L, k::C8, k::C8L);
    case 5:  return rot(v, -k::S8, -k::S8L, k::C8, k::C8L);
    case 7:  return rot(v, -k::C8, -k::C8L, k::S8, k::S8L);
    case 9:  return rot(v, -k::C8, -k::C8L, -k::S8, -k::S8L);
    case 11: return rot(v, -k::S8, -k::S8L, -k::C8, -k::C8L);
    case 13: return rot(v, k::S8, k::S8L, -k::C8, -k::C8L);
    default: return rot(v, k::C8, k::C8L, -k::S8, -k::S8L);
  }
}

// ---------------------------------------------------------------- small DFTs
// Forward DFTs, W_R = exp(-2 pi i / R).
template <int R> struct Dft;

template <> struct Dft<2> {
  template <typename C> __device__ __forceinline__ static void run(C* v, const C*, const C*, int) {
    C a = v[0], b = v[1];
    v[0] = cadd(a, b); v[1] = csub(a, b);
  }
};

template <> struct Dft<4> {
  template <typename C> __device__ __forceinline__ static void run(C* v, const C*, const C*, int) {
    C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    C t2 = cadd(v[1], v[3]), t3 = cmi(csub(v[1], v[3]));
    v[0] = cadd(t0, t2); v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3); v[3] = csub(t1, t3);
  }
};

template <> struct Dft<3> {
  template <typename C> __device__ __forceinline__ static void run(C* v, const C*, const C*, int) {
    using R = decltype(v[0].x);
    C s = cadd(v[1], v[2]), d = csub(v[1], v[2]);
    C a = mk(v[0].x - R(0.5) * s.x, v[0].y - R(0.5) * s.y);
    C r = mk(kmul(d.y, K<R>::H3, K<R>::H3L), kmul(-d.x, K<R>::H3, K<R>::H3L));  // -i sin(2pi/3) d
    v[0] = cadd(v[0], s); v[1] = cadd(a, r); v[2] = csub(a, r);
  }
};

template <> struct Dft<5> {
  template <typename C> __device__ __forceinline__ static void run(C* v, const C*, const C*, int) {
    using R = decltype(v[0].x);
    using k = K<R>;
    C a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
    C a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
    C x0 = v[0];
    C p1 = mk(x0.x + kmul(a1.x, k::C1, k::C1L) + kmul(a2.x, k::C2, k::C2L),
              x0.y + kmul(a1.y, k::C1, k::C1L) + kmul(a2.y, k::C2, k::C2L));
    C p2 = mk(x0.x + kmul(a1.x, k::C2, k::C2L) + kmul(a2.x, k::C1, k::C1L),
              x0.y + kmul(a1.y, k::C2, k::C2L) + kmul(a2.y, k::C1, k::C1L));
    C q1 = cmi(mk(kmul(b1.x, k::S1, k::S1L) + kmul(b2.x, k::S2, k::S2L),
                  kmul(b1.y, k::S1, k::S1L) + kmul(b2.y, k::S2, k::S2L)));
    C q2 = cmi(mk(kmul(b1.x, k::S2, k::S2L) - kmul(b2.x, k::S1, k::S1L),
                  kmul(b1.y, k::S2, k::S2L) - kmul(b2.y, k::S1, k::S1L)));
    v[0] = cadd(x0, cadd(a1, a2));
    v[1] = cadd(p1, q1); v[4] = csub(p1, q1);
    v[2] = cadd(p2, q2); v[3] = csub(p2, q2);
  }
};

// R = R1*R2 from two smaller DFTs: n = R2*n1 + n2, k = k1 + R1*k2.
template <int R1, int R2> struct DftSplit {
  template <typename C> __device__ __forceinline__ static void run(C* v, const C* tw, const C* twl, int unused) {
    using Rl = decltype(v[0].x);
    constexpr int RR = R1 * R2;
    C y[R2][R1];
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) {
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) y[n2][n1] = v[R2 * n1 + n2];
      Dft<R1>::run(y[n2], tw, twl, unused);
#pragma unroll
      for (int k1 = 1; k1 < R1; ++k1) {
        if (n2 == 0) continue;
        // W_RR^(n2 k1) = W_16^(q), RR in {8, 16}
        y[n2][k1] = mul_w16(y[n2][k1], (16 / RR) * ((n2 * k1) % RR));
      }
    }
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
      C z[R2];
#pragma unroll
      for (int n2 = 0; n2 < R2; ++n2) z[n2] = y[n2][k1];
      Dft<R2>::run(z, tw, twl, unused);
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) v[k1 + R1 * k2] = z[k2];
    }
  }
};

// ---- compile-time roots for composite radices other than 8 and 16
// cos and sin of 2 pi e / rr evaluated at compile time: exact quadrant and
// half-quadrant reduction in integers, then Taylor series to x^23 on |t| <= pi/4.
__host__ __device__ constexpr double cx_taylor_sin(double x) {
  double t = x, s = x;
  for (int k = 1; k < 12; ++k) { t *= -x * x / ((2.0 * k) * (2.0 * k + 1.0)); s += t; }
  return s;
}
__host__ __device__ constexpr double cx_taylor_cos(double x) {
  double t = 1.0, s = 1.0;
  for (int k = 1; k < 12; ++k) { t *= -x * x / ((2.0 * k - 1.0) * (2.0 * k)); s += t; }
  return s;
}
struct CxCS { double c, s; };
__host__ __device__ constexpr CxCS cx_root(int e, int rr) {
  const double half_pi = 1.57079632679489661923;
  e = ((e % rr) + rr) % rr;
  const int q = (4 * e) / rr, r = 4 * e - q * rr;
  double cc = 0.0, ss = 0.0;
  if (2 * r <= rr) {
    const double t = half_pi * r / rr;
    cc = cx_taylor_cos(t); ss = cx_taylor_sin(t);
  } else {
    const double t = half_pi * (rr - r) / rr;
    cc = cx_taylor_sin(t); ss = cx_taylor_cos(t);
  }
  if (q == 0) return CxCS{cc, ss};
  if (q == 1) return CxCS{-ss, cc};
  if (q == 2) return CxCS{-cc, -ss};
  return CxCS{ss, -cc};
}

// v * W_RR^E, W_RR = exp(-2 pi i / RR); constants split hi + lo for complex64
template <int RR, int E, typename C> __device__ __forceinline__ C mul_root(C v) {
  using R = decltype(v.x);
  constexpr int e = ((E % RR) + RR) % RR;
  if constexpr (e == 0) {
    return v;
  } else if constexpr (4 * e == RR) {
    return cmi(v);
  } else if constexpr (2 * e == RR) {
    return mk(-v.x, -v.y);
  } else if constexpr (4 * e == 3 * RR) {
    return mk(-v.y, v.x);
  } else {
    constexpr CxCS w = cx_root(e, RR);
    constexpr R ch = (R)w.c, sh = (R)w.s;
    constexpr R cl = (R)(w.c - (double)ch), sl = (R)(w.s - (double)sh);
    return rot(v, ch, cl, sh, sl);
  }
}

template <int B, int E> struct SFor {
  template <typename F> __device__ __forceinline__ static void run(F&& f) {
    if constexpr (B < E) {
      f(std::integral_constant<int, B>{});
      SFor<B + 1, E>::run(f);
    }
  }
};

// R = R1*R2 from two smaller DFTs with compile-time twiddles W_R^(n2 k1).
template <int R1, int R2> struct DftSplitG {
  template <typename C> __device__ __forceinline__ static void run(C* v, const C* tw, const C* twl, int unused) {
    C y[R2][R1];
    SFor<0, R2>::run([&](auto n2c) {
      constexpr int n2 = decltype(n2c)::value;
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) y[n2][n1] = v[R2 * n1 + n2];
      Dft<R1>::run(y[n2], tw, twl, unused);
      SFor<1, R1>::run([&](auto k1c) {
        constexpr int k1 = decltype(k1c)::value;
        y[n2][k1] = mul_root<R1 * R2, n2 * k1>(y[n2][k1]);
      });
    });
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
      C z[R2];
#pragma unroll
      for (int n2 = 0; n2 < R2; ++n2) z[n2] = y[n2][k1];
      Dft<R2>::run(z, tw, twl, unused);
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) v[k1 + R1 * k2] = z[k2];
    }
  }
};

template <> struct Dft<8>  : DftSplit<4, 2> {};
template <> struct Dft<16> : DftSplit<4, 4> {};
template <> struct Dft<6>  : DftSplitG<3, 2> {};
template <> struct Dft<10> : DftSplitG<5, 2> {};
template <> struct Dft<12> : DftSplitG<4, 3> {};
template <> struct Dft<32> : DftSplitG<4, 8> {};

// Generic odd prime radix (7, 11, 13): direct O(R^2) DFT, W_R^e read from the
// length-n twiddle table (tw[j] = W_n^j) at stride n/R.
template <int R> struct DftDirect {
  template <typename C> __device__ __forceinline__ static void run(C* v, const C* tw, const C* twl, int n_over_r) {
    C w[R], wl[R];
#pragma unroll
    for (int j = 0; j < R; ++j) { w[j] = tw[j * n_over_r]; wl[j] = twl[j * n_over_r]; }
    C out[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
      C acc = v[0];
#pragma unroll
      for (int m = 1; m < R; ++m) acc = cadd(acc, twmul(v[m], w[(m * k) % R], wl[(m * k) % R]));
      out[k] = acc;
    }
#pragma unroll
    for (int k = 0; k < R; ++k) v[k] = out[k];
  }
};
template <> struct Dft<7>  : DftDirect<7> {};
template <> struct Dft<11> : DftDirect<11> {};
template <> struct Dft<13> : DftDirect<13> {};

// ---------------------------------------------------------------- one pass
template <int R, int EPT, typename C>
__device__ __forceinline__ void stockham_pass(C* __restrict__ s, const C* __restrict__ tw,
                                              const C* __restrict__ twl, int n, int p, int nl, int sn,
                                              int sl) {
  constexpr int Q = (EPT + R - 1) / R;
  const int nb = n / R;
  const int total = nb * nl;
  const int tws = n / (p * R);
  const int nt = blockDim.x;
  C v[Q][R];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int b = threadIdx.x + q * nt;
    if (b < total) {
      const int l = b % nl, i = b / nl;
      const C* src = s + l * sl + i * sn;
#pragma unroll
      for (int m = 0; m < R; ++m) v[q][m] = src[m * nb * sn];
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int b = threadIdx.x + q * nt;
    if (b < total) {
      const int l = b % nl, i = b / nl;
      const int k = i % p;
      if (k != 0) {
        const int step = k * tws;
#pragma unroll
        for (int m = 1; m < R; ++m) v[q][m] = twmul(v[q][m], tw[m * step], twl[m * step]);
      }
      Dft<R>::run(v[q], tw, twl, nb);
      C* dst = s + l * sl + ((i - k) * R + k) * sn;
#pragma unroll
      for (int m = 0; m < R; ++m) dst[m * p * sn] = v[q][m];
    }
  }
  __syncthreads();
}

struct PassPlan {
  int n;
  int npass;
  int radix[12];
};

// Forward FFT of every line of the tile (natural order in and out).
// GEN = false: radices 2, 3, 4, 5, 8, 16 only (the register budget of the
// common sizes); GEN = true adds the direct odd-prime radices 7, 11, 13.
template <int EPT, bool GEN, typename C>
__device__ __forceinline__ void fft_lines(C* s, const C* tw, const C* twl, const PassPlan& pp, int nl, int sn,
                                          int sl) {
  int p = 1;
  for (int q = 0; q < pp.npass; ++q) {
    const int r = pp.radix[q];
    switch (r) {
      case 16: stockham_pass<16, EPT>(s, tw, twl, pp.n, p, nl, sn, sl); break;
      case 8:  stockham_pass<8, EPT>(s, tw, twl, pp.n, p, nl, sn, sl); break;
      case 4:  stockham_pass<4, EPT>(s, tw, twl, pp.n, p, nl, sn, sl); break;
      case 2:  stockham_pass<2, EPT>(s, tw, twl, pp.n, p, nl, sn, sl); break;
      case 3:  stockham_pass<3, EPT>(s, tw, twl, pp.n, p, nl, sn, sl); break;
      case 5:  stockham_pass<5, EPT>(s, tw, twl, pp.n, p, nl, sn, sl); break;
      default:
        if constexpr (GEN) {
          if (r == 7) stockham_pass<7, EPT>(s, tw, twl, pp.n, p, nl, sn, sl);
          else if (r == 11) stockham_pass<11, EPT>(s, tw, twl, pp.n, p, nl, sn, sl);
          else stockham_pass<13, EPT>(s, tw, twl, pp.n, p, nl, sn, sl);
        }
        break;
    }
    p *= r;
  }
}

}  // namespace gpe
