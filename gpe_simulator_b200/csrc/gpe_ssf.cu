// gpe_ssf.cu -- plans, launch sequences and the C ABI (include/gpe_ssf.h).
#include <cuda.h>
#include "../../include/gpe_ssf.h"
#include "gpe_sweep.h"
#include "gpe_fast.cuh"

namespace gpe {
cudaError_t launch_fast_tma(int n, int ax, const Phys& ph, const Sweep& sw, const FastOps& op,
                            const CUtensorMap& map, cudaStream_t st);
template <typename R>
cudaError_t launch_fast(int n, int ax, const Phys& ph, const Sweep& sw, const FastOps& op, cudaStream_t st);
template <typename R>
cudaError_t launch_fast_batch(int n, int ax, const Phys* phs, const Sweep* sws, int count, const FastOps& op,
                              cudaStream_t st);
template <typename R>
cudaError_t launch_plane(int n, int mz, const Phys& ph, const Sweep& sw, const PlaneJob& job, cudaStream_t st);
}

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace gpe;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

}  // namespace

namespace gpe {
void set_last_error(const std::string& msg) { g_err = msg; }
}  // namespace gpe

namespace {

#define CU(call)                                                                            \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess) {                                                                \
      if (e_ == cudaErrorMemoryAllocation) return fail(GPE_ERR_OOM, cudaGetErrorString(e_)); \
      return fail(GPE_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));        \
    }                                                                                       \
  } while (0)

#define TRY(x) do { int r_ = (x); if (r_ != GPE_OK) return r_; } while (0)

// Host evaluation of a potential program (same semantics as eval_program).
double host_eval(const std::vector<double>& prog, double x, double y, double z, double t) {
  double st[GPE_STACK_MAX];
  int sp = 0;
  for (size_t pc = 0; pc < prog.size();) {
    const int op = (int)prog[pc++];
    switch (op) {
      case GPE_OP_CONST: st[sp++] = prog[pc++]; break;
      case GPE_OP_X: st[sp++] = x; break;
      case GPE_OP_Y: st[sp++] = y; break;
      case GPE_OP_Z: st[sp++] = z; break;
      case GPE_OP_T: st[sp++] = t; break;
      case GPE_OP_ADD: --sp; st[sp - 1] = st[sp - 1] + st[sp]; break;
      case GPE_OP_SUB: --sp; st[sp - 1] = st[sp - 1] - st[sp]; break;
      case GPE_OP_MUL: --sp; st[sp - 1] = st[sp - 1] * st[sp]; break;
      case GPE_OP_DIV: --sp; st[sp - 1] = st[sp - 1] / st[sp]; break;
      case GPE_OP_POW: --sp; st[sp - 1] = std::pow(st[sp - 1], st[sp]); break;
      case GPE_OP_NEG: st[sp - 1] = -st[sp - 1]; break;
      case GPE_OP_SIN: st[sp - 1] = std::sin(st[sp - 1]); break;
      case GPE_OP_COS: st[sp - 1] = std::cos(st[sp - 1]); break;
      case GPE_OP_TAN: st[sp - 1] = std::tan(st[sp - 1]); break;
      case GPE_OP_EXP: st[sp - 1] = std::exp(st[sp - 1]); break;
      case GPE_OP_SQRT: st[sp - 1] = std::sqrt(st[sp - 1]); break;
      case GPE_OP_TANH: st[sp - 1] = std::tanh(st[sp - 1]); break;
      case GPE_OP_ABS: st[sp - 1] = std::fabs(st[sp - 1]); break;
      case GPE_OP_LOG: st[sp - 1] = std::log(st[sp - 1]); break;
      default: break;
    }
  }
  return sp ? st[0] : 0.0;
}

// ---- dynamic potentials on the register-resident sweeps
// A dynamic potential V(x, y, z, t) whose additive terms do not depend on z is
// constant along every z-line at a given time, so the z sweeps can take it per
// line instead of per point (a stirring beam rotating in the x-y plane is of
// this form).  The bytecode is read back into a tree; every subexpression that
// depends on t alone becomes a slot (evaluated on the host in FP64 once per
// launch, at each half-step time), constant subexpressions are folded, and
// powers 2 become squares.  What remains is a short program in (x, y) that the
// z sweeps evaluate once per line in FP64.
struct ExprNode {
  int op = 0;
  double val = 0.0;
  int a = -1, b = -1;
  unsigned vars = 0;   // 1 x, 2 y, 4 z, 8 t
};

bool expr_tree(const std::vector<double>& prog, std::vector<ExprNode>& nodes, int& root) {
  std::vector<int> st;
  for (size_t pc = 0; pc < prog.size();) {
    ExprNode nd;
    nd.op = (int)prog[pc++];
    switch (nd.op) {
      case GPE_OP_CONST: nd.val = prog[pc++]; break;
      case GPE_OP_X: nd.vars = 1; break;
      case GPE_OP_Y: nd.vars = 2; break;
      case GPE_OP_Z: nd.vars = 4; break;
      case GPE_OP_T: nd.vars = 8; break;
      case GPE_OP_ADD: case GPE_OP_SUB: case GPE_OP_MUL: case GPE_OP_DIV: case GPE_OP_POW:
        if (st.size() < 2) return false;
        nd.b = st.back(); st.pop_back();
        nd.a = st.back(); st.pop_back();
        nd.vars = nodes[nd.a].vars | nodes[nd.b].vars;
        break;
      default:   // unary
        if (st.empty()) return false;
        nd.a = st.back(); st.pop_back();
        nd.vars = nodes[nd.a].vars;
        break;
    }
    nodes.push_back(nd);
    st.push_back((int)nodes.size() - 1);
  }
  if (st.size() != 1) return false;
  root = st[0];
  return true;
}

void expr_emit_plain(const std::vector<ExprNode>& nodes, int i, std::vector<double>& out) {
  const ExprNode& nd = nodes[i];
  if (nd.a >= 0) expr_emit_plain(nodes, nd.a, out);
  if (nd.b >= 0) expr_emit_plain(nodes, nd.b, out);
  out.push_back((double)nd.op);
  if (nd.op == GPE_OP_CONST) out.push_back(nd.val);
}

// Residual line program of node i: t-only subtrees become slots, constant
// subtrees constants, x^2 a square.  False when the slot budget runs out.
bool expr_emit_line(const std::vector<ExprNode>& nodes, int i, std::vector<double>& out,
                    std::vector<std::vector<double>>& slots) {
  const ExprNode& nd = nodes[i];
  if (nd.vars == 0 && nd.op != GPE_OP_CONST) {
    std::vector<double> sub;
    expr_emit_plain(nodes, i, sub);
    out.push_back(GPE_OP_CONST);
    out.push_back(host_eval(sub, 0.0, 0.0, 0.0, 0.0));
    return true;
  }
  if (nd.vars == 8) {
    if ((int)slots.size() == GPE_LINE_SLOTS) return false;
    std::vector<double> sub;
    expr_emit_plain(nodes, i, sub);
    slots.push_back(sub);
    out.push_back((double)(OP_SLOT0 + (int)slots.size() - 1));
    return true;
  }
  if (nd.op == GPE_OP_POW && nodes[nd.b].vars == 0) {
    std::vector<double> sub;
    expr_emit_plain(nodes, nd.b, sub);
    if (host_eval(sub, 0.0, 0.0, 0.0, 0.0) == 2.0) {
      if (!expr_emit_line(nodes, nd.a, out, slots)) return false;
      out.push_back((double)OP_SQR);
      return true;
    }
  }
  if (nd.a >= 0 && !expr_emit_line(nodes, nd.a, out, slots)) return false;
  if (nd.b >= 0 && !expr_emit_line(nodes, nd.b, out, slots)) return false;
  out.push_back((double)nd.op);
  if (nd.op == GPE_OP_CONST) out.push_back(nd.val);
  return true;
}

// Line form of a dynamic program: true (with `line` and `slots` filled) when no
// additive term depends on z.
bool dynamic_line_form(const std::vector<double>& prog, std::vector<double>& line,
                       std::vector<std::vector<double>>& slots) {
  std::vector<ExprNode> nodes;
  int root = -1;
  if (!expr_tree(prog, nodes, root)) return false;
  // signed top-level terms of the sum
  std::vector<std::pair<int, int>> terms;
  std::vector<std::pair<int, int>> todo{{root, 1}};
  while (!todo.empty()) {
    const auto [i, sign] = todo.back();
    todo.pop_back();
    const ExprNode& nd = nodes[i];
    if (nd.op == GPE_OP_ADD) { todo.push_back({nd.b, sign}); todo.push_back({nd.a, sign}); }
    else if (nd.op == GPE_OP_SUB) { todo.push_back({nd.b, -sign}); todo.push_back({nd.a, sign}); }
    else if (nd.op == GPE_OP_NEG) todo.push_back({nd.a, -sign});
    else terms.push_back({i, sign});
  }
  line.clear();
  slots.clear();
  bool first = true;
  for (const auto& [i, sign] : terms) {
    if (nodes[i].vars & 4) return false;
    if (!expr_emit_line(nodes, i, line, slots)) return false;
    if (sign < 0) line.push_back(GPE_OP_NEG);
    if (!first) line.push_back(GPE_OP_ADD);
    first = false;
  }
  return (int)line.size() <= GPE_PROGRAM_MAX;
}

// Validate a program: known opcodes, operands present, stack within bounds, one result.
bool check_program(const double* p, int len, std::string& why) {
  if (len == 0) return true;
  if (!p || len < 0 || len > GPE_PROGRAM_MAX) { why = "program length out of range"; return false; }
  int sp = 0;
  for (int pc = 0; pc < len;) {
    const double opd = p[pc++];
    const int op = (int)opd;
    if ((double)op != opd) { why = "non-integer opcode"; return false; }
    int pop = 0, push = 1;
    switch (op) {
      case GPE_OP_CONST:
        if (pc >= len) { why = "constant without operand"; return false; }
        ++pc; pop = 0; break;
      case GPE_OP_X: case GPE_OP_Y: case GPE_OP_Z: case GPE_OP_T: pop = 0; break;
      case GPE_OP_ADD: case GPE_OP_SUB: case GPE_OP_MUL: case GPE_OP_DIV: case GPE_OP_POW: pop = 2; break;
      case GPE_OP_NEG: case GPE_OP_SIN: case GPE_OP_COS: case GPE_OP_TAN: case GPE_OP_EXP:
      case GPE_OP_SQRT: case GPE_OP_TANH: case GPE_OP_ABS: case GPE_OP_LOG: pop = 1; break;
      default: why = "unknown opcode"; return false;
    }
    if (sp < pop) { why = "stack underflow"; return false; }
    sp = sp - pop + push;
    if (sp > GPE_STACK_MAX - 1) { why = "expression too deep"; return false; }
  }
  if (sp != 1) { why = "program must leave exactly one value"; return false; }
  return true;
}

bool factorize(int n, PassPlan& pp) {
  pp.n = n;
  pp.npass = 0;
  int m = n, twos = 0;
  while (m % 2 == 0) { m /= 2; ++twos; }
  std::vector<int> r;
  // powers of two: radix 16 where possible; remainders balanced with 8/4/2
  int t = twos;
  if (t % 4 == 1 && t >= 5) { r.push_back(8); r.push_back(4); t -= 5; }
  else if (t % 4 == 1) { r.push_back(2); t -= 1; }
  else if (t % 4 == 2) { r.push_back(4); t -= 2; }
  else if (t % 4 == 3) { r.push_back(8); t -= 3; }
  while (t >= 4) { r.push_back(16); t -= 4; }
  const int odd[] = {3, 5, 7, 11, 13};
  for (int p : odd)
    while (m % p == 0) { r.push_back(p); m /= p; }
  if (m != 1) return false;
  if ((int)r.size() > 12) return false;
  for (size_t i = 0; i < r.size(); ++i) pp.radix[i] = r[i];
  pp.npass = (int)r.size();
  return true;
}

}  // namespace

// ---------------------------------------------------------------- small kernels
namespace gpe {

// d_v[idx] = general static program + Re(staticV) (or the real array), precision R;
// d_im[idx] = Im(staticV) for a complex staticV (real time).
template <typename R>
__global__ void k_build_static(int n, const double* x, const double* prog, int len, const void* v,
                               int kind, R* out_re, R* out_im) {
  const long long m = (long long)n * n * n;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < m;
       idx += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(idx % n), j = (int)((idx / n) % n), i = (int)(idx / ((long long)n * n));
    double re = 0.0, im = 0.0;
    if (len) re += eval_program(prog, len, x[i], x[j], x[k], 0.0);
    if (kind == GPE_V_REAL64) re += ((const double*)v)[idx];
    if (kind == GPE_V_CPLX128) {
      const double2 c = ((const double2*)v)[idx];
      re += c.x;
      im = c.y;
    }
    if (out_re) out_re[idx] = (R)re;
    if (out_im) out_im[idx] = (R)im;
  }
}

// Sum per-block diagnostic partials in a fixed order: out[0..3] = sums of pa
// columns 0..2 and pb column 3 (the shell bins out[4 + b] come from k_finish_hist).
__global__ void k_finish_diag(const double* pa, int na, const double* pb, int nb, double* out) {
  __shared__ Acc sh[32 * 4];
  Acc a[4];
  for (int b = threadIdx.x; b < na; b += blockDim.x) {
    a[0].add(pa[b * 4 + 0]);
    a[1].add(pa[b * 4 + 1]);
    a[2].add(pa[b * 4 + 2]);
  }
  for (int b = threadIdx.x; b < nb; b += blockDim.x) a[3].add(pb[b * 4 + 3]);
  block_merge<4>(a, sh);
  if (threadIdx.x == 0)
    for (int v = 0; v < 4; ++v) out[v] = a[v].value();
}

// k-space sums of a spectrum passed in by the caller (no transform): sum k^2 |f|^2
// (the reference's get_E, gpe/helper.py:135-140) into partial[block * 4 + 3] and,
// with `hist`, the block's shell histogram of |f|^2 (gpe/nk_extraction.py:5-21)
// into hist[block][nbins].  Each warp walks whole rows (x, y) with its lanes
// along z, so the row's k_x^2 + k_y^2 and indices are computed once per row.
template <typename C>
__global__ void __launch_bounds__(256) k_kspace(const C* __restrict__ f, int n, const double* __restrict__ k,
                                                double* __restrict__ partial, double* __restrict__ hist,
                                                int nbins, double shell_w) {
  extern __shared__ double sh_hist[];
  __shared__ Acc red[32];
  if (hist) {
    for (int b = threadIdx.x; b < nbins; b += blockDim.x) sh_hist[b] = 0.0;
    __syncthreads();
  }
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  double e = 0.0;
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n * n; r += warps) {
    const int i = r / n, j = r - i * n;
    const double kx = k[i], ky = k[j];
    const C* row = f + (long long)r * n;
    for (int z = lane; z < n; z += 32) {
      const double kk = kk_ref(kx, ky, k[z]);
      const C v = row[z];
      const double w = (double)v.x * v.x + (double)v.y * v.y;
      e = fma(kk, w, e);
      if (hist) {
        int sh = (int)floor(sqrt(kk) / shell_w + 0.5);
        sh = min(sh, nbins - 1);
        atomicAdd(sh_hist + sh, w);
      }
    }
  }
  Acc a[1];
  a[0].add(e);
  block_merge<1>(a, red);
  if (threadIdx.x == 0) partial[(long long)blockIdx.x * 4 + 3] = a[0].value();
  if (hist) {
    __syncthreads();
    for (int b = threadIdx.x; b < nbins; b += blockDim.x) hist[(long long)blockIdx.x * nbins + b] = sh_hist[b];
  }
}

// Shell histograms: block `bin` sums that bin over the nb per-tile histograms
// (threads stride over the tiles with compensation, merged in a fixed order)
// into out[4 + bin].
__global__ void k_finish_hist(const double* hist, int nb, int nbins, double* out) {
  __shared__ Acc sh[32];
  const int bin = blockIdx.x;
  Acc a[1];
  for (int b = threadIdx.x; b < nb; b += blockDim.x) a[0].add(hist[(long long)b * nbins + bin]);
  block_merge<1>(a, sh);
  if (threadIdx.x == 0) out[4 + bin] = a[0].value();
}

// Lagged renormalisation of a whole state with the pending scale (the
// arithmetic of PW_SCALE: complex64 times (float)(1/sqrt N), complex128 divided
// by sqrt N), elementwise: a thread takes 4 elements, a warp 4 runs of 32.
template <typename R>
__device__ __forceinline__ void scale_state(typename Cx<R>::T* psi, long long count, const double* scale) {
  using C = typename Cx<R>::T;
  const long long e0 = (long long)blockIdx.x * blockDim.x * 4 + threadIdx.x;
  C v[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const long long e = e0 + (long long)q * blockDim.x;
    v[q] = e < count ? psi[e] : mk((R)0, (R)0);
  }
  if (sizeof(R) == 4) {
    const R f = (R)__ldcg(scale + 1);
#pragma unroll
    for (int q = 0; q < 4; ++q) { v[q].x *= f; v[q].y *= f; }
  } else {
    const double d = __ldcg(scale);
#pragma unroll
    for (int q = 0; q < 4; ++q) { v[q].x = (R)((double)v[q].x / d); v[q].y = (R)((double)v[q].y / d); }
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const long long e = e0 + (long long)q * blockDim.x;
    if (e < count) psi[e] = v[q];
  }
}

template <typename R>
__global__ void __launch_bounds__(256) k_scale(Sweep sw, long long count) {
  scale_state<R>((typename Cx<R>::T*)sw.dst, count, sw.scale);
}

// batched: blockIdx.y selects the instance
template <typename R>
__global__ void __launch_bounds__(256) k_scale_batch(const Sweep* __restrict__ sws, long long count) {
  if (batch_frozen(sws[blockIdx.y].live)) return;
  scale_state<R>((typename Cx<R>::T*)sws[blockIdx.y].dst, count, sws[blockIdx.y].scale);
}

// Batched finish: block b sums the partials of instance jobs[b] into out[4*index].
// The constants give the instance's energy from its sums (as diag_scalars does).
struct DiagJob {
  const double* pa;
  const double* pb;
  int na, nb, index;
  int imag;                       // imaginary-time instance (takes part in convergence)
  double ckin, dx3, inv_m, beta;
};

// Real-time batch groups: member q takes entry tick[q] of the call's time table
// (host-computed, FP64: t_mid of the step and the beam centres at it, t at the
// step's end and the centres there) into its z sweeps' and diagnostics'
// descriptors, then advances.
__global__ void k_batch_clock(Sweep* sws, int m, const double* times, int* tick, int r1, int r2, int rd) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= m) return;
  const double* e = times + ((size_t)tick[q] * m + q) * 6;
  Sweep* a = sws + (size_t)r1 * m + q;
  Sweep* b = sws + (size_t)r2 * m + q;
  Sweep* d = sws + (size_t)rd * m + q;
  a->t1 = b->t1 = e[0];
  a->bc1x = b->bc1x = e[1];
  a->bc1y = b->bc1y = e[2];
  d->t1 = e[3];
  d->bc1x = e[4];
  d->bc1y = e[5];
  tick[q] += 1;
}

__global__ void k_finish_diag_batch(const DiagJob* jobs, double* out) {
  __shared__ Acc sh[32 * 4];
  const DiagJob j = jobs[blockIdx.x];
  Acc a[4];
  for (int b = threadIdx.x; b < j.na; b += blockDim.x) {
    a[0].add(j.pa[b * 4 + 0]);
    a[1].add(j.pa[b * 4 + 1]);
    a[2].add(j.pa[b * 4 + 2]);
  }
  for (int b = threadIdx.x; b < j.nb; b += blockDim.x) a[3].add(j.pb[b * 4 + 3]);
  block_merge<4>(a, sh);
  if (threadIdx.x == 0)
    for (int v = 0; v < 4; ++v) out[4 * j.index + v] = a[v].value();
}

// On-device convergence of batched imaginary-time solves, after each chunk's
// diagnostics: a live instance advances its step count by the chunk, forms its
// energy from the finished sums exactly as the host does (same operations, no
// contraction), and freezes when |E - E_last| / (chunk |E|) < tol (false for a
// NaN E_last: no first-check convergence) or its steps reach max_steps.  The
// rule of Batch.solve and of one solve at a time (checks every `chunk` steps).
__global__ void k_batch_converge(const DiagJob* jobs, int njobs, const double* sums, int chunk, double tol,
                                 long long max_steps, int* live, long long* steps, double* e_last) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= njobs) return;
  const DiagJob jb = jobs[j];
  const int i = jb.index;
  if (!jb.imag || !live[i]) return;
  const double* h = sums + 4 * i;
  const double e_kin = __dmul_rn(__dmul_rn(__dmul_rn(jb.ckin, h[3]), jb.dx3), jb.inv_m);
  const double e_pot = __dmul_rn(h[1], jb.dx3);
  const double e_int = __dmul_rn(__dmul_rn(__dmul_rn(0.5, jb.beta), h[2]), jb.dx3);
  const double e = __dadd_rn(__dadd_rn(e_kin, e_pot), e_int);
  const long long s = steps[i] + chunk;
  const double rate = __ddiv_rn(fabs(__dsub_rn(e, e_last[i])), __dmul_rn((double)chunk, fabs(e)));
  steps[i] = s;
  e_last[i] = e;
  if (rate < tol || s >= max_steps) live[i] = 0;
}

__global__ void k_fill_int(int* a, int n, int v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}

// ---------------------------------------------------------------- image projections
// The image outputs of the reference's save_outputs (gpe/save.py:59-90); out
// arrays are n x n, row-major, at fftshifted indices for the momentum images.
__device__ __forceinline__ int fftshift_index(int i, int n) { return (i + n / 2) % n; }

// one warp per (a, b) line along the contiguous axis: sum |v|^2 over it, and the
// element at `pick` of the line; `shift` selects fftshifted output indices
template <typename C>
__global__ void k_proj_lines(const C* __restrict__ f, int n, double col_scale, double pick_scale, int pick,
                             bool shift, double* __restrict__ col, double* __restrict__ sel,
                             double* __restrict__ sel_phase) {
  const long long line = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / 32;
  const int lane = threadIdx.x & 31;
  if (line >= (long long)n * n) return;
  const int a = (int)(line / n), b = (int)(line % n);
  const C* row = f + line * n;
  double s = 0.0;
  for (int z = lane; z < n; z += 32) s += (double)row[z].x * row[z].x + (double)row[z].y * row[z].y;
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) {
    const long long o = shift ? (long long)fftshift_index(a, n) * n + fftshift_index(b, n) : line;
    if (col) col[o] = s * col_scale;
    const C v = row[pick];
    if (sel) sel[o] = ((double)v.x * v.x + (double)v.y * v.y) * pick_scale;
    if (sel_phase) sel_phase[o] = atan2((double)v.y, (double)v.x);
  }
}

// one thread per (b, c): sum |f[a][b][c]|^2 over the slowest axis a, and a = 0
template <typename C>
__global__ void k_proj_slow(const C* __restrict__ f, int n, double col_scale, double pick_scale,
                            double* __restrict__ col, double* __restrict__ sel) {
  const long long bc = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (bc >= (long long)n * n) return;
  const long long plane = (long long)n * n;
  double s = 0.0;
  for (int a = 0; a < n; ++a) {
    const C v = f[a * plane + bc];
    s += (double)v.x * v.x + (double)v.y * v.y;
  }
  const int b = (int)(bc / n), c = (int)(bc % n);
  const long long o = (long long)fftshift_index(b, n) * n + fftshift_index(c, n);
  if (col) col[o] = s * col_scale;
  if (sel) { const C v = f[bc]; sel[o] = ((double)v.x * v.x + (double)v.y * v.y) * pick_scale; }
}

// phase = NaN where the slice density is below 1e-12 of its maximum (one block)
__global__ void k_phase_mask(const double* __restrict__ dens, double* __restrict__ phase, long long count) {
  __shared__ double sm[32];
  double m = 0.0;
  for (long long i = threadIdx.x; i < count; i += blockDim.x) m = fmax(m, dens[i]);
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x / 32] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < blockDim.x / 32 ? sm[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) sm[0] = m;
  }
  __syncthreads();
  const double thr = sm[0] * 1e-12;
  for (long long i = threadIdx.x; i < count; i += blockDim.x)
    if (!(dens[i] > thr)) phase[i] = nan("");
}

}  // namespace gpe

// ---------------------------------------------------------------- the plan
struct gpe_plan {
  int n = 0, dtype = 0, kind = 0;
  double beta = 0, dt = 0, ckin = 1, dx = 0;
  size_t csize = 8;                // bytes per complex element
  std::vector<double> x, k;
  std::vector<double> prog_static_g, prog_dyn;
  std::vector<double> prog_line;                   // dynamic potential per z-line (register-resident sweeps)
  std::vector<std::vector<double>> slot_progs;     // its time-dependent subexpressions (host, per launch)
  PassPlan pp{};
  Phys ph{};
  int lt_z = 1, lt_yx = 16;
  bool gen = false;                // grid size needs the odd-prime radices 7/11/13
  bool fast = false;               // register-resident sweeps exist for this n
  bool plane = false;              // y and z sweeps fused per x-plane (opt-in; complex64, n = 128, 256)
  bool tma = false;                // plain y/x sweeps stage their pencils by TMA (opt-in; complex64, n = 128, 256)
  // tensor maps of recently swept arrays: base address -> maps of y and x tiles
  struct TmaMaps { const void* base; CUtensorMap map[2]; };
  TmaMaps tma_cache[4] = {};
  int tma_next = 0;
  bool pdl_chain = false;          // inside a step sequence: sweeps may launch programmatically
  bool pdl_prev = false;           // a sweep of the current sequence has been launched
  int ept = 16;                    // elements per thread of the sweep family
  int nbins = 0;
  double shell_w = 0;
  std::vector<long long> counts;
  // device buffers
  double* d_x = nullptr;
  double* d_k = nullptr;
  double2* d_kin = nullptr;
  double* d_kth = nullptr;
  void* d_vax = nullptr;
  void* d_vre = nullptr;
  void* d_vim = nullptr;
  double* d_prog_g = nullptr;
  double* d_dyn = nullptr;
  double* d_line = nullptr;
  void* d_ltab = nullptr;          // [2][n*n] per-line dynamic potential (line form), precision of psi
  void* d_tw = nullptr;
  double* d_partial = nullptr;   // 2 areas of 4*max_tiles doubles
  unsigned* d_ticket = nullptr;
  unsigned* d_plane = nullptr;   // plane-fused launches: ticket, finished blocks, per (plane, stage) counts
  double* d_scale = nullptr;     // [sqrtN, 1/sqrtN, N, ...]
  int* d_status = nullptr;
  double* d_hist = nullptr;
  double* d_out = nullptr;       // diag results [4 + nbins]
  void* d_work = nullptr;        // diagnostic FFT scratch (size of psi), lazily
  double* d_proj = nullptr;      // image projections: 7 n x n arrays, lazily
  int max_tiles = 0;
  // launch accounting and optional per-launch timing (events around each sweep)
  long long launches = 0;
  bool prof = false;
  struct Rec { int ax; cudaEvent_t a, b; };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> pool;
};

namespace {

int tiles_of(const gpe_plan* p, int ax) {
  const int n = p->n;
  if (ax == AX_Z) return (n * n + p->lt_z - 1) / p->lt_z;
  return n * ((n + p->lt_yx - 1) / p->lt_yx);
}

// Plan-owned pointers of a generic sweep and its launch geometry.
template <typename R>
int sweep_geometry(const gpe_plan* p, int ax, Sweep& sw, int& tiles, int& threads, size_t& smem) {
  using C = typename Cx<R>::T;
  const int n = p->n;
  sw.pp = p->pp;
  sw.tw = p->d_tw;
  sw.tw_lo = (const char*)p->d_tw + (size_t)n * sizeof(C);
  sw.ticket = p->d_ticket;
  sw.scale = p->d_scale;
  sw.status = p->d_status;
  sw.nbins = p->nbins;
  sw.shell_w = p->shell_w;
  int lt = ax == AX_Z ? p->lt_z : p->lt_yx;
  sw.lt = lt;
  sw.tiles_per_row = (n + p->lt_yx - 1) / p->lt_yx;
  tiles = tiles_of(p, ax);
  const int pitch = ax == AX_Z ? ((n & 1) ? n : n + 1) : lt;
  const int tile_elems = ax == AX_Z ? lt * pitch : n * lt;
  const int E = n * lt;
  threads = (E + p->ept - 1) / p->ept;
  threads = ((threads + 31) / 32) * 32;
  if (threads < 32) threads = 32;
  if (threads > 512) return fail(GPE_ERR_UNSUPPORTED, "tile too large");
  smem = (size_t)(2 * n + tile_elems) * sizeof(C) + 32 * 4 * sizeof(Acc) + (size_t)p->nbins * sizeof(double);
  if (smem > 200 * 1024) return fail(GPE_ERR_UNSUPPORTED, "tile does not fit in shared memory");
  return GPE_OK;
}

template <typename R>
int launch(gpe_plan* p, int ax, Sweep sw, cudaStream_t st) {
  int tiles = 0, threads = 0;
  size_t smem = 0;
  TRY(sweep_geometry<R>(p, ax, sw, tiles, threads, smem));
  CU(launch_sweep<R>(ax, p->gen, p->ph, sw, tiles, threads, smem, st));
  return GPE_OK;
}

cudaEvent_t pooled_event(gpe_plan* p) {
  if (!p->pool.empty()) {
    cudaEvent_t e = p->pool.back();
    p->pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Centres of the stirring beam at the sweep's half-step times t1, t2: the angle
// th(t) = omega (m^2/(2 t_ramp) + t - m), m = min(t, t_ramp) (linear ramp of the
// angular rate), in FP64 once per launch.
void beam_centres(const gpe_plan* p, Sweep& sw) {
  sw.bc1x = sw.bc1y = sw.bc2x = sw.bc2y = 0.0;
  if (!(p->kind == GPE_REAL && p->ph.beam)) return;
  const Phys& ph = p->ph;
  auto centre = [&](double t, double& cx, double& cy) {
    double th;
    if (ph.beam_t_ramp > 0.0) {
      const double m = std::min(t, ph.beam_t_ramp);
      th = ph.beam_omega * (m * m / (2.0 * ph.beam_t_ramp) + t - m);
    } else {
      th = ph.beam_omega * t;
    }
    cx = ph.beam_radius * std::cos(th);
    cy = ph.beam_radius * std::sin(th);
  };
  centre(sw.t1, sw.bc1x, sw.bc1y);
  centre(sw.t2, sw.bc2x, sw.bc2y);
}

// The line table of the next z sweep: the line program's slot values at t1
// (and t2) in FP64 on the host, then one thread per z-line and time on the
// device.  Inside a step sequence it is a programmatic dependent of the sweep
// before it, and the z sweep after it is one of it.
int line_table(gpe_plan* p, double t1, double t2, bool two, cudaStream_t st) {
  LineSlots sl;
  memset(&sl, 0, sizeof(sl));
  for (size_t k = 0; k < p->slot_progs.size(); ++k) {
    sl.s1[k] = host_eval(p->slot_progs[k], 0.0, 0.0, 0.0, t1);
    sl.s2[k] = host_eval(p->slot_progs[k], 0.0, 0.0, 0.0, t2);
  }
  const long long count = (two ? 2LL : 1LL) * p->n * p->n;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)((count + 255) / 256));
  cfg.blockDim = dim3(256);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = p->pdl_chain && p->pdl_prev && !p->prof ? 1 : 0;
  const double* prog = p->d_line;
  const int len = (int)p->prog_line.size();
  const cudaError_t e =
      p->dtype == GPE_C64
          ? cudaLaunchKernelEx(&cfg, k_line_table<float>, prog, len, (const double*)p->d_x, p->n, sl,
                               (float*)p->d_ltab, two ? 1 : 0)
          : cudaLaunchKernelEx(&cfg, k_line_table<double>, prog, len, (const double*)p->d_x, p->n, sl,
                               (double*)p->d_ltab, two ? 1 : 0);
  if (e != cudaSuccess) return fail(GPE_ERR_CUDA, std::string("line table: ") + cudaGetErrorString(e));
  ++p->launches;
  p->pdl_prev = p->pdl_chain;
  return GPE_OK;
}

bool needs_lines(int mode) { return mode == FM_Z1 || mode == FM_Z2 || mode == FM_Z21 || mode == FM_DIAGR; }

int sweep(gpe_plan* p, int ax, const Sweep& sw_in, cudaStream_t st) {
  Sweep sw = sw_in;
  beam_centres(p, sw);
  gpe_plan::Rec r{ax, nullptr, nullptr};
  if (p->prof) {
    r.a = pooled_event(p);
    r.b = pooled_event(p);
    CU(cudaEventRecord(r.a, st));
  }
  const int rc = p->dtype == GPE_C64 ? launch<float>(p, ax, sw, st) : launch<double>(p, ax, sw, st);
  if (rc == GPE_OK) ++p->launches;
  if (p->prof) {
    CU(cudaEventRecord(r.b, st));
    p->recs.push_back(r);
  }
  return rc;
}

// cuTensorMapEncodeTiled from the driver, through the runtime's entry-point
// query (no link-time dependency on libcuda); null when unavailable.
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)f;
  }
  return fn;
}

// Tensor maps of the n^3 complex64 array at `base` (8-byte elements, dims z, y,
// x innermost first): y tiles are boxes {L, n, 1}, x tiles {L, 1, n}, L the
// sweeps' lines per tile.  Null when the array cannot be staged (base not
// 16-byte aligned, encoder missing).
const CUtensorMap* tma_maps(gpe_plan* p, const void* base, int fax) {
  const int which = fax == FY ? 0 : 1;
  for (auto& c : p->tma_cache)
    if (c.base == base) return &c.map[which];
  EncodeTiledFn enc = encode_tiled();
  if (!enc || ((uintptr_t)base & 15u)) return nullptr;
  const cuuint64_t n = (cuuint64_t)p->n;
  const cuuint64_t dims[3] = {n, n, n};
  const cuuint64_t strides[2] = {n * 8, n * n * 8};
  const cuuint32_t lt = (cuuint32_t)fast_lines(p->n, 4);
  const cuuint32_t boxes[2][3] = {{lt, (cuuint32_t)n, 1}, {lt, 1, (cuuint32_t)n}};
  const cuuint32_t estr[3] = {1, 1, 1};
  gpe_plan::TmaMaps& c = p->tma_cache[p->tma_next];
  for (int a = 0; a < 2; ++a) {
    const CUresult r = enc(&c.map[a], CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, const_cast<void*>(base), dims, strides,
                           boxes[a], estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
      c.base = nullptr;
      return nullptr;
    }
  }
  c.base = base;
  p->tma_next = (p->tma_next + 1) % 4;
  return &c.map[which];
}

// Register-resident sweep (n with a fast split); same accounting as sweep().
int fsweep(gpe_plan* p, int ax, Sweep sw, const FastOps& op, cudaStream_t st) {
  beam_centres(p, sw);
  if (p->d_ltab && needs_lines(op.mode)) TRY(line_table(p, sw.t1, sw.t2, op.mode == FM_Z21, st));
  sw.pp = p->pp;
  sw.tw = p->d_tw;
  sw.tw_lo = (const char*)p->d_tw + (size_t)p->n * p->csize;
  sw.ticket = p->d_ticket;
  sw.scale = p->d_scale;
  sw.status = p->d_status;
  gpe_plan::Rec r{ax, nullptr, nullptr};
  if (p->prof) {
    r.a = pooled_event(p);
    r.b = pooled_event(p);
    CU(cudaEventRecord(r.a, st));
  }
  const int fax = ax == AX_Z ? FZ : ax == AX_Y ? FY : FX;
  FastOps o = op;
  o.pdl = p->pdl_chain && p->pdl_prev && !p->prof ? 1 : 0;
  p->pdl_prev = p->pdl_chain;
  const CUtensorMap* map = p->tma && o.mode == FM_PLAIN && fax != FZ ? tma_maps(p, sw.src, fax) : nullptr;
  const cudaError_t e = map ? launch_fast_tma(p->n, fax, p->ph, sw, o, *map, st)
                        : p->dtype == GPE_C64 ? launch_fast<float>(p->n, fax, p->ph, sw, o, st)
                                              : launch_fast<double>(p->n, fax, p->ph, sw, o, st);
  if (e != cudaSuccess) return fail(GPE_ERR_CUDA, std::string("fast sweep: ") + cudaGetErrorString(e));
  ++p->launches;
  if (p->prof) {
    CU(cudaEventRecord(r.b, st));
    p->recs.push_back(r);
  }
  return GPE_OK;
}

// One plane-fused launch: up to three consecutive y/z sweeps of psi (in place),
// stage `zstage` a z sweep of mode `mz`, the others y sweeps.  Recorded as a z
// launch in the per-axis profile.
int psweep(gpe_plan* p, void* psi, int mz, const FastOps* ops, int nstage, int zstage, double t1, double t2,
           cudaStream_t st) {
  Sweep sw;
  memset(&sw, 0, sizeof(sw));
  sw.src = psi;
  sw.dst = psi;
  sw.t1 = t1;
  sw.t2 = t2;
  beam_centres(p, sw);
  if (p->d_ltab) TRY(line_table(p, t1, t2, mz == FM_Z21, st));
  sw.partial = p->d_partial;
  sw.pp = p->pp;
  sw.tw = p->d_tw;
  sw.tw_lo = (const char*)p->d_tw + (size_t)p->n * p->csize;
  sw.ticket = p->d_ticket;
  sw.scale = p->d_scale;
  sw.status = p->d_status;
  PlaneJob job;
  memset(&job, 0, sizeof(job));
  for (int i = 0; i < nstage; ++i) job.op[i] = ops[i];
  job.nstage = nstage;
  job.zstage = zstage;
  job.ctr = p->d_plane;
  gpe_plan::Rec r{AX_Z, nullptr, nullptr};
  if (p->prof) {
    r.a = pooled_event(p);
    r.b = pooled_event(p);
    CU(cudaEventRecord(r.a, st));
  }
  p->pdl_prev = false;   // the sweep after a persistent plane launch starts normally
  const cudaError_t e = launch_plane<float>(p->n, mz, p->ph, sw, job, st);
  if (e != cudaSuccess) return fail(GPE_ERR_CUDA, std::string("plane sweep: ") + cudaGetErrorString(e));
  ++p->launches;
  if (p->prof) {
    CU(cudaEventRecord(r.b, st));
    p->recs.push_back(r);
  }
  return GPE_OK;
}

FastOps mk_ops(int mode, int inv1 = 0, int invm = 0, int scale = 0, int norm = 0) {
  FastOps o;
  o.mode = mode; o.inv1 = inv1; o.invm = invm; o.scale = scale; o.norm = norm; o.pdl = 0; o.pf = 0;
  return o;
}

// Scope of one step sequence: its register-resident sweeps after the first are
// launched as programmatic dependents of the sweep before (they read only plan
// constants until their grid-dependency wait).
struct PdlChain {
  gpe_plan* p;
  explicit PdlChain(gpe_plan* q) : p(q) { p->pdl_chain = true; p->pdl_prev = false; }
  ~PdlChain() { p->pdl_chain = false; p->pdl_prev = false; }
};

Sweep mk_sweep(const void* src, void* dst) {
  Sweep s;
  memset(&s, 0, sizeof(s));
  s.src = src;
  s.dst = dst;
  return s;
}

// reference: t = i*dt (gpe/launch.py:10), t_mid = t + dt/2 (gpe/make_propagator.py:94)
double t_mid_host(const gpe_plan* p, long long step) { return (double)step * p->dt + p->dt / 2; }


// Norm of psi into d_scale (sqrtN, 1/sqrtN, N) via a no-store sweep.
int norm_sweep(gpe_plan* p, const void* psi, cudaStream_t st) {
  Sweep s = mk_sweep(psi, nullptr);
  s.post = PW_NORM;
  s.partial = p->d_partial;
  return sweep(p, AX_Z, s, st);
}

int scale_sweep(gpe_plan* p, void* psi, cudaStream_t st) {
  Sweep s = mk_sweep(psi, psi);
  s.scale = p->d_scale;
  const long long count = (long long)p->n * p->n * p->n;
  const unsigned blocks = (unsigned)((count + 1023) / 1024);
  if (p->dtype == GPE_C64) k_scale<float><<<blocks, 256, 0, st>>>(s, count);
  else k_scale<double><<<blocks, 256, 0, st>>>(s, count);
  CU(cudaGetLastError());
  ++p->launches;
  return GPE_OK;
}

int ensure_work(gpe_plan* p) {
  if (p->d_work) return GPE_OK;
  const size_t bytes = (size_t)p->n * p->n * p->n * p->csize;
  CU(cudaMalloc(&p->d_work, bytes));
  return GPE_OK;
}

int ensure_hist(gpe_plan* p) {
  if (p->d_hist) return GPE_OK;
  // per-tile histograms of the generic or the register-resident x sweep
  const size_t bytes = (size_t)p->max_tiles * p->nbins * sizeof(double);
  CU(cudaMalloc(&p->d_hist, bytes));
  return GPE_OK;
}

int fill_plan(gpe_plan* p, const gpe_desc* d) {
  const int n = d->n;
  if (n < 2 || n > 1024) return fail(GPE_ERR_UNSUPPORTED, "n must be in [2, 1024]");
  if (!factorize(n, p->pp)) return fail(GPE_ERR_UNSUPPORTED, "n has a prime factor larger than 13");
  if (d->dtype != GPE_C64 && d->dtype != GPE_C128) return fail(GPE_ERR_ARG, "dtype must be GPE_C64 or GPE_C128");
  if (d->kind != GPE_IMAGINARY && d->kind != GPE_REAL) return fail(GPE_ERR_ARG, "kind must be imaginary or real");
  if (!d->x_array || !d->k_array) return fail(GPE_ERR_ARG, "x_array and k_array are required");
  if (!std::isfinite(d->beta) || !std::isfinite(d->dt) || !std::isfinite(d->kinetic_coeff))
    return fail(GPE_ERR_ARG, "beta, dt and kinetic_coeff must be finite");
  std::string why;
  const double* progs[] = {d->static_x, d->static_y, d->static_z, d->static_g, d->dynamic_g};
  const int lens[] = {d->static_x_len, d->static_y_len, d->static_z_len, d->static_g_len, d->dynamic_g_len};
  for (int q = 0; q < 5; ++q)
    if (!check_program(progs[q], lens[q], why)) return fail(GPE_ERR_ARG, "potential program: " + why);
  if (d->kind == GPE_IMAGINARY && (d->dynamic_g_len || d->beam_enabled || d->k_cut_enabled))
    return fail(GPE_ERR_ARG, "imaginary time takes no time-dependent potential, beam or cutoff");
  p->n = n;
  p->dtype = d->dtype;
  p->kind = d->kind;
  p->beta = d->beta;
  p->dt = d->dt;
  p->ckin = d->kinetic_coeff;
  p->csize = d->dtype == GPE_C64 ? 8 : 16;
  p->x.assign(d->x_array, d->x_array + n);
  p->k.assign(d->k_array, d->k_array + n);
  p->dx = p->x[1] - p->x[0];
  if (d->static_g_len) p->prog_static_g.assign(d->static_g, d->static_g + d->static_g_len);
  if (d->dynamic_g_len) p->prog_dyn.assign(d->dynamic_g, d->dynamic_g + d->dynamic_g_len);
  // kernel family and tiles: at most 512 threads x ept elements per tile;
  // 128-byte rows for y/x tiles, ~4096 elements per z tile
  for (int q = 0; q < p->pp.npass; ++q)
    if (p->pp.radix[q] > 5 && p->pp.radix[q] != 8 && p->pp.radix[q] != 16) p->gen = true;
  p->ept = p->gen ? 8 : 16;
  // register-resident sweeps: n = 32, 48, 64, 96, 128, 160, 256; potentials from tables (no per-point program)
  // (complex64 plans that evaluate the local factor in FP64 use the generic sweeps,
  // which carry that variant; keeping it out of the register-resident kernels keeps
  // their register budget)
  // a dynamic potential stays on them when none of its terms depends on z (line form)
  const bool line_ok = d->dynamic_g_len == 0 || dynamic_line_form(p->prog_dyn, p->prog_line, p->slot_progs);
  p->fast = (n == 32 || n == 48 || n == 64 || n == 96 || n == 128 || n == 160 || n == 256 ||
             (n == 512 && d->dtype == GPE_C64)) &&
            d->generic_only != 1 && line_ok && !(d->local_fp64 && d->dtype == GPE_C64) &&
            !d->exact_local;
  if (!p->fast) { p->prog_line.clear(); p->slot_progs.clear(); }
  p->plane = p->fast && d->dtype == GPE_C64 && (n == 128 || n == 256) && d->generic_only == 3;
  p->tma = p->fast && d->dtype == GPE_C64 && (n == 128 || n == 256) && d->generic_only == 4;
  const int emax = 512 * p->ept;
  p->lt_yx = std::max(1, std::min(d->dtype == GPE_C64 ? 16 : 8, emax / n));
  p->lt_z = std::max(1, std::min(n * n, std::min(4096, emax) / n));
  // shells (reference gpe/nk_extraction.py:19-21)
  const double dk = std::fabs(p->k[1] - p->k[0]);
  if (d->nk_bins > 0) {
    if (d->nk_bins < 2) return fail(GPE_ERR_ARG, "nk_bins must be >= 2");
    p->nbins = d->nk_bins;
    p->shell_w = std::sqrt(3.0) * (n / 2) * dk / (p->nbins - 1);
  } else {
    p->nbins = (int)std::floor(std::sqrt(3.0) * (n / 2) + 0.5) + 1;
    p->shell_w = dk;
  }
  p->counts.assign(p->nbins, 0);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j)
      for (int l = 0; l < n; ++l) {
        const double kk = p->k[i] * p->k[i] + p->k[j] * p->k[j] + p->k[l] * p->k[l];
        int s = (int)std::floor(std::sqrt(kk) / p->shell_w + 0.5);
        p->counts[std::min(s, p->nbins - 1)]++;
      }
  p->max_tiles = std::max(tiles_of(p, AX_Z), tiles_of(p, AX_X));
  return GPE_OK;
}

template <typename R>
int upload_tables(gpe_plan* p, const gpe_desc* d) {
  const int n = p->n;
  // twiddles W_n^j = exp(-2 pi i j/n), computed in long double and rounded once
  std::vector<typename Cx<R>::T> tw(n), twl(n);
  for (int j = 0; j < n; ++j) {
    const long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)j / (long double)n;
    const long double c = cosl(a), s = sinl(a);
    tw[j].x = (R)(double)c;
    tw[j].y = (R)(double)s;
    // residuals: complex64 applies twiddles as hi + lo (exact value and modulus)
    twl[j].x = sizeof(R) == 4 ? (R)(double)(c - (long double)tw[j].x) : (R)0;
    twl[j].y = sizeof(R) == 4 ? (R)(double)(s - (long double)tw[j].y) : (R)0;
  }
  CU(cudaMalloc(&p->d_tw, 2 * n * sizeof(tw[0])));
  CU(cudaMemcpy(p->d_tw, tw.data(), n * sizeof(tw[0]), cudaMemcpyHostToDevice));
  CU(cudaMemcpy((char*)p->d_tw + n * sizeof(tw[0]), twl.data(), n * sizeof(tw[0]), cudaMemcpyHostToDevice));
  // static axis potentials
  std::vector<R> vax(3 * n, (R)0);
  const double* ap[] = {d->static_x, d->static_y, d->static_z};
  const int al[] = {d->static_x_len, d->static_y_len, d->static_z_len};
  for (int a = 0; a < 3; ++a) {
    if (!al[a]) continue;
    std::vector<double> prog(ap[a], ap[a] + al[a]);
    for (int i = 0; i < n; ++i) {
      const double c = p->x[i];
      vax[a * n + i] = (R)host_eval(prog, a == 0 ? c : 0.0, a == 1 ? c : 0.0, a == 2 ? c : 0.0, 0.0);
    }
  }
  CU(cudaMalloc(&p->d_vax, 3 * n * sizeof(R)));
  CU(cudaMemcpy(p->d_vax, vax.data(), 3 * n * sizeof(R), cudaMemcpyHostToDevice));
  return GPE_OK;
}

int build_static(gpe_plan* p, const void* v, int v_kind, cudaStream_t st) {
  const size_t m = (size_t)p->n * p->n * p->n;
  const size_t rs = p->dtype == GPE_C64 ? 4 : 8;
  const bool need_re = !p->prog_static_g.empty() || v_kind != GPE_V_NONE;
  const bool need_im = v_kind == GPE_V_CPLX128 && p->kind == GPE_REAL;
  if (need_re && !p->d_vre) CU(cudaMalloc(&p->d_vre, m * rs));
  if (need_im && !p->d_vim) CU(cudaMalloc(&p->d_vim, m * rs));
  if (!need_re && p->d_vre) { CU(cudaFree(p->d_vre)); p->d_vre = nullptr; }
  if (!need_im && p->d_vim) { CU(cudaFree(p->d_vim)); p->d_vim = nullptr; }
  p->ph.vre = p->d_vre;
  p->ph.vim = p->d_vim;
  if (!need_re && !need_im) return GPE_OK;
  const int len = (int)p->prog_static_g.size();
  if (p->dtype == GPE_C64)
    k_build_static<float><<<1184, 256, 0, st>>>(p->n, p->d_x, p->d_prog_g, len, v, v_kind,
                                               (float*)p->d_vre, (float*)p->d_vim);
  else
    k_build_static<double><<<1184, 256, 0, st>>>(p->n, p->d_x, p->d_prog_g, len, v, v_kind,
                                                (double*)p->d_vre, (double*)p->d_vim);
  CU(cudaGetLastError());
  return GPE_OK;
}

void free_plan(gpe_plan* p) {
  for (auto& r : p->recs) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
  for (auto e : p->pool) cudaEventDestroy(e);
  void* bufs[] = {p->d_x, p->d_k, p->d_kin, p->d_kth, p->d_vax, p->d_vre, p->d_vim, p->d_prog_g, p->d_dyn, p->d_line, p->d_ltab,
                  p->d_tw, p->d_partial, p->d_ticket, p->d_scale, p->d_status, p->d_hist, p->d_out,
                  p->d_work, p->d_plane, p->d_proj};
  for (void* b : bufs)
    if (b) cudaFree(b);
  delete p;
}

int create(const gpe_desc* d, gpe_plan** out) {
  gpe_plan* p = new gpe_plan();
  int rc = fill_plan(p, d);
  if (rc != GPE_OK) { delete p; return rc; }
  const int n = p->n;
  CU(cudaMalloc(&p->d_x, n * sizeof(double)));
  CU(cudaMemcpy(p->d_x, p->x.data(), n * sizeof(double), cudaMemcpyHostToDevice));
  CU(cudaMalloc(&p->d_k, n * sizeof(double)));
  CU(cudaMemcpy(p->d_k, p->k.data(), n * sizeof(double), cudaMemcpyHostToDevice));
  // kinetic factors per axis: exp(-i ckin k^2 dt) or exp(-ckin k^2 dt)
  std::vector<double2> kin(n);
  for (int i = 0; i < n; ++i) {
    const double ph = p->ckin * p->k[i] * p->k[i] * p->dt;
    kin[i] = p->kind == GPE_IMAGINARY ? make_double2(std::exp(-ph), 0.0)
                                      : make_double2(std::cos(ph), -std::sin(ph));
  }
  CU(cudaMalloc(&p->d_kin, n * sizeof(double2)));
  CU(cudaMemcpy(p->d_kin, kin.data(), n * sizeof(double2), cudaMemcpyHostToDevice));
  std::vector<double> kth(n);
  for (int i = 0; i < n; ++i) kth[i] = p->ckin * p->k[i] * p->k[i] * p->dt;
  CU(cudaMalloc(&p->d_kth, n * sizeof(double)));
  CU(cudaMemcpy(p->d_kth, kth.data(), n * sizeof(double), cudaMemcpyHostToDevice));
  rc = p->dtype == GPE_C64 ? upload_tables<float>(p, d) : upload_tables<double>(p, d);
  if (rc != GPE_OK) { free_plan(p); return rc; }
  if (!p->prog_static_g.empty()) {
    CU(cudaMalloc(&p->d_prog_g, p->prog_static_g.size() * sizeof(double)));
    CU(cudaMemcpy(p->d_prog_g, p->prog_static_g.data(), p->prog_static_g.size() * sizeof(double),
                  cudaMemcpyHostToDevice));
  }
  if (!p->prog_dyn.empty()) {
    CU(cudaMalloc(&p->d_dyn, p->prog_dyn.size() * sizeof(double)));
    CU(cudaMemcpy(p->d_dyn, p->prog_dyn.data(), p->prog_dyn.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  if (!p->prog_line.empty()) {
    CU(cudaMalloc(&p->d_line, p->prog_line.size() * sizeof(double)));
    CU(cudaMemcpy(p->d_line, p->prog_line.data(), p->prog_line.size() * sizeof(double), cudaMemcpyHostToDevice));
    CU(cudaMalloc(&p->d_ltab, 2 * (size_t)n * n * (p->dtype == GPE_C64 ? 4 : 8)));
  }
  CU(cudaMalloc(&p->d_partial, 2 * 4 * (size_t)p->max_tiles * sizeof(double)));
  CU(cudaMalloc(&p->d_ticket, sizeof(unsigned)));
  CU(cudaMemset(p->d_ticket, 0, sizeof(unsigned)));
  if (p->plane) {
    CU(cudaMalloc(&p->d_plane, (2 + 3 * (size_t)n) * sizeof(unsigned)));
    CU(cudaMemset(p->d_plane, 0, (2 + 3 * (size_t)n) * sizeof(unsigned)));
  }
  CU(cudaMalloc(&p->d_scale, 4 * sizeof(double)));
  const double one[4] = {1.0, 1.0, 1.0, 0.0};
  CU(cudaMemcpy(p->d_scale, one, sizeof(one), cudaMemcpyHostToDevice));
  CU(cudaMalloc(&p->d_status, sizeof(int)));
  CU(cudaMemset(p->d_status, 0, sizeof(int)));
  CU(cudaMalloc(&p->d_out, (4 + p->nbins) * sizeof(double)));
  Phys& ph = p->ph;
  ph.kind = p->kind;
  ph.beta = p->beta;
  ph.dt = p->dt;
  ph.ckin = p->ckin;
  ph.inv_m = 1.0 / ((double)n * n * n);
  ph.dx3 = p->dx * p->dx * p->dx;
  ph.x = p->d_x;
  ph.k = p->d_k;
  ph.kin = p->d_kin;
  ph.kth = p->d_kth;
  ph.vax = p->d_vax;
  ph.dyn = p->d_dyn;
  ph.dyn_len = (int)p->prog_dyn.size();
  ph.ltab = p->d_ltab;
  ph.beam = d->beam_enabled ? 1 : 0;
  ph.beam_amp = d->beam_amp;
  ph.beam_inv_w2 = d->beam_enabled ? 1.0 / (d->beam_width * d->beam_width) : 0.0;
  ph.beam_radius = d->beam_radius;
  ph.beam_omega = d->beam_omega;
  ph.beam_t_ramp = d->beam_t_ramp;
  ph.kcut = d->k_cut_enabled ? 1 : 0;
  ph.kcut2 = d->k_cut * d->k_cut;
  ph.local_fp64 = d->local_fp64 ? 1 : 0;
  ph.exact_local = d->exact_local ? 1 : 0;
  rc = build_static(p, nullptr, GPE_V_NONE, 0);
  if (rc != GPE_OK) { free_plan(p); return rc; }
  CU(cudaDeviceSynchronize());
  *out = p;
  return GPE_OK;
}

// One Strang step (5 sweeps) whose half-steps use time `t` (t_mid);
// `scaled` = psi carries a pending renormalisation.
int strang_step(gpe_plan* p, void* psi, double t, bool scaled, cudaStream_t st) {
  const bool imag = p->kind == GPE_IMAGINARY;
  Sweep s = mk_sweep(psi, psi);
  s.pre = PW_HALF1 | (scaled ? PW_SCALE : 0u);
  s.fft1 = 1;
  s.t1 = t;
  TRY(sweep(p, AX_Z, s, st));
  s = mk_sweep(psi, psi);
  s.fft1 = 1;
  TRY(sweep(p, AX_Y, s, st));
  s = mk_sweep(psi, psi);
  s.fft1 = 1;
  s.mid = PW_KIN | PW_CONJ_LAST;
  s.fft2 = 1;
  s.post = PW_CONJ_FIRST;
  TRY(sweep(p, AX_X, s, st));
  s = mk_sweep(psi, psi);
  s.pre = PW_CONJ_LAST;
  s.fft1 = 1;
  s.post = PW_CONJ_FIRST;
  TRY(sweep(p, AX_Y, s, st));
  s = mk_sweep(psi, psi);
  s.pre = PW_CONJ_LAST;
  s.fft1 = 1;
  s.post = PW_CONJ_FIRST | PW_INVM | PW_HALF1 | (imag ? PW_NORM : 0u);
  s.t1 = t;
  s.partial = p->d_partial;
  TRY(sweep(p, AX_Z, s, st));
  return GPE_OK;
}

// Fast path, 5 sweeps: Z(half, fwd) Y(fwd) X(fwd, kin, inv) Y(inv) Z(inv, 1/M, half [, norm]).
// With `fuse_next`, the last sweep also applies the next step's half-step and
// forward z transform (real time), so the next step starts at its Y sweep.
int fast_front(gpe_plan* p, void* psi, double t, bool scaled, cudaStream_t st) {
  Sweep s = mk_sweep(psi, psi);
  s.t1 = t;
  return fsweep(p, AX_Z, s, mk_ops(FM_Z1, 0, 0, scaled ? 1 : 0), st);
}

int fast_middle(gpe_plan* p, void* psi, cudaStream_t st) {
  Sweep s = mk_sweep(psi, psi);
  TRY(fsweep(p, AX_Y, s, mk_ops(FM_PLAIN), st));
  TRY(fsweep(p, AX_X, s, mk_ops(FM_XKIN), st));
  return fsweep(p, AX_Y, s, mk_ops(FM_PLAIN, 1), st);
}

int fast_back(gpe_plan* p, void* psi, double t, double t_next, bool fuse_next, cudaStream_t st) {
  const bool imag = p->kind == GPE_IMAGINARY;
  Sweep s = mk_sweep(psi, psi);
  s.t1 = t;
  s.t2 = t_next;
  s.partial = p->d_partial;
  if (fuse_next) return fsweep(p, AX_Z, s, mk_ops(FM_Z21), st);
  return fsweep(p, AX_Z, s, mk_ops(FM_Z2, 0, 0, 0, imag ? 1 : 0), st);
}

int fft3d(gpe_plan* p, const void* in, void* out, bool inverse, cudaStream_t st) {
  if (p->fast) {
    Sweep s = mk_sweep(in, out);
    if (!inverse) {
      TRY(fsweep(p, AX_Z, s, mk_ops(FM_PLAIN), st));
      s.src = out;
      TRY(fsweep(p, AX_Y, s, mk_ops(FM_PLAIN), st));
      return fsweep(p, AX_X, s, mk_ops(FM_PLAIN), st);
    }
    TRY(fsweep(p, AX_X, s, mk_ops(FM_PLAIN, 1), st));
    s.src = out;
    TRY(fsweep(p, AX_Y, s, mk_ops(FM_PLAIN, 1), st));
    return fsweep(p, AX_Z, s, mk_ops(FM_PLAIN, 1, 1), st);
  }
  if (!inverse) {
    Sweep s = mk_sweep(in, out);
    s.fft1 = 1;
    TRY(sweep(p, AX_Z, s, st));
    s.src = out;
    TRY(sweep(p, AX_Y, s, st));
    TRY(sweep(p, AX_X, s, st));
    return GPE_OK;
  }
  Sweep s = mk_sweep(in, out);
  s.pre = PW_CONJ_LAST;
  s.fft1 = 1;
  s.post = PW_CONJ_FIRST;
  TRY(sweep(p, AX_X, s, st));
  s.src = out;
  TRY(sweep(p, AX_Y, s, st));
  s.post = PW_CONJ_FIRST | PW_INVM;
  TRY(sweep(p, AX_Z, s, st));
  return GPE_OK;
}

// k-space reductions of a spectrum `f` (no FFT): partial area B + histogram.
// k-space reductions of a spectrum `f` (no FFT): per-block sums of k^2 |f|^2
// (+ shell histograms) into partial area B; `nb` = the blocks to finish.
int kspace_reduce(gpe_plan* p, const void* f, bool hist, int& nb, cudaStream_t st) {
  TRY(ensure_hist(p));
  // at most max_tiles blocks (the partial and histogram areas), 4 per SM
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    CU(cudaGetDevice(&dev));
    CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  }
  const size_t smem = hist ? (size_t)p->nbins * sizeof(double) : 0;
  if (smem > 48 * 1024) return fail(GPE_ERR_UNSUPPORTED, "too many n(k) bins for the shared histogram");
  nb = std::max(1, std::min(p->max_tiles, std::min(4 * sms, (p->n * p->n + 7) / 8)));
  double* part = p->d_partial + 4 * (size_t)p->max_tiles;
  double* h = hist ? p->d_hist : nullptr;
  if (p->dtype == GPE_C64)
    k_kspace<float2><<<nb, 256, smem, st>>>((const float2*)f, p->n, p->d_k, part, h, p->nbins, p->shell_w);
  else
    k_kspace<double2><<<nb, 256, smem, st>>>((const double2*)f, p->n, p->d_k, part, h, p->nbins, p->shell_w);
  CU(cudaGetLastError());
  ++p->launches;
  return GPE_OK;
}

int finish_diag(gpe_plan* p, int na, int nb, bool hist, std::vector<double>& host, cudaStream_t st) {
  k_finish_diag<<<1, 256, 0, st>>>(p->d_partial, na, p->d_partial + 4 * (size_t)p->max_tiles, nb, p->d_out);
  if (hist) k_finish_hist<<<p->nbins, 256, 0, st>>>(p->d_hist, nb, p->nbins, p->d_out);
  CU(cudaGetLastError());
  host.assign(4 + p->nbins, 0.0);
  CU(cudaMemcpyAsync(host.data(), p->d_out, host.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  return GPE_OK;
}

// The three diagnostic sweeps of psi at time t (real-space sums in the z sweep
// writing the partial transform to the plan's work buffer, k-space sums and
// shells in the x sweep); results stay on the device until finish_diag.
// Tile counts of the diagnostic z and x sweeps (the partials to finish).
void diag_tiles(const gpe_plan* p, bool fast, int& na, int& nb) {
  if (fast) {
    const int lt = fast_lines(p->n, (int)p->csize / 2);
    na = p->n * p->n / lt;
    nb = p->n * (p->n / lt);
  } else {
    na = tiles_of(p, AX_Z);
    nb = tiles_of(p, AX_X);
  }
}

// The diagnostics run on the register-resident sweeps when the plan has them
// and the shell histogram (if wanted) fits their shared tables region.
bool diag_fast(const gpe_plan* p, bool hist) {
  return p->fast && (!hist || (size_t)p->nbins * sizeof(double) <= fast_tables_bytes_rt(p->n, (int)p->csize / 2));
}

int diag_launch(gpe_plan* p, const void* psi, double t, bool hist, cudaStream_t st) {
  if (diag_fast(p, hist)) {
    Sweep s = mk_sweep(psi, p->d_work);
    s.t1 = t;
    s.partial = p->d_partial;
    TRY(fsweep(p, AX_Z, s, mk_ops(FM_DIAGR), st));
    s = mk_sweep(p->d_work, p->d_work);
    TRY(fsweep(p, AX_Y, s, mk_ops(FM_PLAIN), st));
    s = mk_sweep(p->d_work, nullptr);
    s.partial = p->d_partial + 4 * (size_t)p->max_tiles;
    s.hist = hist ? p->d_hist : nullptr;
    s.nbins = p->nbins;
    s.shell_w = p->shell_w;
    return fsweep(p, AX_X, s, mk_ops(FM_DIAGK), st);
  }
  Sweep s = mk_sweep(psi, p->d_work);
  s.pre = PW_DIAG_R;
  s.t1 = t;
  s.fft1 = 1;
  s.partial = p->d_partial;
  TRY(sweep(p, AX_Z, s, st));
  s = mk_sweep(p->d_work, p->d_work);
  s.fft1 = 1;
  TRY(sweep(p, AX_Y, s, st));
  s = mk_sweep(p->d_work, nullptr);
  s.fft1 = 1;
  s.post = PW_DIAG_K;
  s.partial = p->d_partial + 4 * (size_t)p->max_tiles;
  s.hist = p->d_hist;
  return sweep(p, AX_X, s, st);
}

// Lz of psi (reference gpe/helper.py:143-156).  By Parseval along each axis the
// reference's slab sums become two k-space sums of the z-transformed state F_z:
//   Lz = dx^3/n^2 [ sum x k_y |FFT_y F_z|^2 - sum y k_x |FFT_x F_z|^2 ],
// one forward z sweep into the work buffer and two read-only sweeps (x, y) of it;
// the per-tile partials are summed on the host in tile order (deterministic).
int angular_momentum(gpe_plan* p, const void* psi, double* lz, cudaStream_t st) {
  TRY(ensure_work(p));
  Sweep s = mk_sweep(psi, p->d_work);
  s.fft1 = 1;
  TRY(sweep(p, AX_Z, s, st));
  s = mk_sweep(p->d_work, nullptr);
  s.fft1 = 1;
  s.post = PW_LZ_X;
  s.partial = p->d_partial;
  TRY(sweep(p, AX_X, s, st));
  s = mk_sweep(p->d_work, nullptr);
  s.fft1 = 1;
  s.post = PW_LZ_Y;
  s.partial = p->d_partial + 4 * (size_t)p->max_tiles;
  TRY(sweep(p, AX_Y, s, st));
  const int nx = tiles_of(p, AX_X), ny = tiles_of(p, AX_Y);
  std::vector<double> hx(4 * (size_t)nx), hy(4 * (size_t)ny);
  CU(cudaMemcpyAsync(hx.data(), p->d_partial, hx.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  CU(cudaMemcpyAsync(hy.data(), p->d_partial + 4 * (size_t)p->max_tiles, hy.size() * sizeof(double),
                     cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  // compensated sums in tile order
  auto csum = [](const std::vector<double>& v, int count) {
    double sum = 0.0, c = 0.0;
    for (int b = 0; b < count; ++b) {
      const double y = v[4 * (size_t)b + 3] - c, t = sum + y;
      c = (t - sum) - y;
      sum = t;
    }
    return sum;
  };
  const double n2 = (double)p->n * p->n;
  *lz = (csum(hy, ny) - csum(hx, nx)) / n2 * p->ph.dx3;
  return GPE_OK;
}

// The selected image projections of psi (GPE_PROJ_* bits, reference
// gpe/save.py:59-90) into `out` (host), n*n doubles per selected image in bit order.
template <typename R>
int projections(gpe_plan* p, const void* psi, unsigned which, double* out, cudaStream_t st) {
  using C = typename Cx<R>::T;
  const int n = p->n;
  const long long nn = (long long)n * n;
  if (!p->d_proj) CU(cudaMalloc(&p->d_proj, 7 * nn * sizeof(double)));
  double* img[7];
  for (int i = 0; i < 7; ++i) img[i] = (which >> i) & 1u ? p->d_proj + i * nn : nullptr;
  const double dx = p->dx, dk = std::fabs(p->k[1] - p->k[0]);
  const double scale = dx * dx * dx / ((double)nn * n * dk * dk * dk);
  const unsigned tof = GPE_PROJ_TOF_XY | GPE_PROJ_TOF_YZ | GPE_PROJ_TOF_SLICE_XY | GPE_PROJ_TOF_SLICE_YZ;
  const int warps_per_block = 8;
  const unsigned lines_grid = (unsigned)((nn + warps_per_block - 1) / warps_per_block);
  if (which & tof) {
    TRY(ensure_work(p));
    TRY(fft3d(p, psi, p->d_work, false, st));
    const C* f = (const C*)p->d_work;
    if (img[0] || img[2])
      k_proj_lines<C><<<lines_grid, 32 * warps_per_block, 0, st>>>(f, n, scale * dk, scale, 0, true, img[0],
                                                                   img[2], nullptr);
    if (img[1] || img[3])
      k_proj_slow<C><<<(unsigned)((nn + 255) / 256), 256, 0, st>>>(f, n, scale * dk, scale, img[1], img[3]);
    CU(cudaGetLastError());
  }
  if (which & (GPE_PROJ_DENSITY_XY | GPE_PROJ_DENSITY_SLICE_XY | GPE_PROJ_PHASE_XY)) {
    double* slice = img[5] ? img[5] : (img[6] ? p->d_proj + 5 * nn : nullptr);
    k_proj_lines<C><<<lines_grid, 32 * warps_per_block, 0, st>>>((const C*)psi, n, dx, 1.0, n / 2, false, img[4],
                                                                 slice, img[6]);
    if (img[6]) k_phase_mask<<<1, 1024, 0, st>>>(slice, img[6], nn);
    CU(cudaGetLastError());
  }
  for (int i = 0, o = 0; i < 7; ++i)
    if (img[i]) {
      CU(cudaMemcpyAsync(out + (size_t)o * nn, img[i], nn * sizeof(double), cudaMemcpyDeviceToHost, st));
      ++o;
    }
  CU(cudaStreamSynchronize(st));
  return GPE_OK;
}

// {N, E_kin, E_pot, E_int, E, mu} from the finished sums h[0..3].
void diag_scalars(const gpe_plan* p, const double* h, double* scalars) {
  const double dx3 = p->ph.dx3;
  const double N = h[0] * dx3;
  const double e_kin = p->ckin * h[3] * dx3 * p->ph.inv_m;
  const double e_pot = h[1] * dx3;
  const double e_int = 0.5 * p->beta * h[2] * dx3;
  scalars[0] = N;
  scalars[1] = e_kin;
  scalars[2] = e_pot;
  scalars[3] = e_int;
  scalars[4] = e_kin + e_pot + e_int;
  scalars[5] = (e_kin + e_pot + 2.0 * e_int) / N;
}

}  // namespace

// ================================================================ C ABI
extern "C" {

int gpe_version(void) { return 1; }

int gpe_last_error(char* buf, size_t len) {
  if (!buf || !len) return (int)g_err.size();
  snprintf(buf, len, "%s", g_err.c_str());
  return (int)g_err.size();
}

int gpe_plan_create(const gpe_desc* desc, gpe_plan** plan) {
  if (!desc || !plan) return fail(GPE_ERR_ARG, "null argument");
  *plan = nullptr;
  return create(desc, plan);
}

int gpe_plan_destroy(gpe_plan* plan) {
  if (!plan) return GPE_OK;
  free_plan(plan);
  return GPE_OK;
}

int gpe_plan_info(const gpe_plan* p, int* n, int* dtype, int* kind, int* nk_bins) {
  if (!p) return fail(GPE_ERR_ARG, "null plan");
  if (n) *n = p->n;
  if (dtype) *dtype = p->dtype;
  if (kind) *kind = p->kind;
  if (nk_bins) *nk_bins = p->nbins;
  return GPE_OK;
}

int gpe_set_static_potential(gpe_plan* p, const void* v, int v_kind, void* stream) {
  if (!p) return fail(GPE_ERR_ARG, "null plan");
  if (v_kind != GPE_V_NONE && v_kind != GPE_V_REAL64 && v_kind != GPE_V_CPLX128)
    return fail(GPE_ERR_ARG, "unknown static potential kind");
  if (v_kind != GPE_V_NONE && !v) return fail(GPE_ERR_ARG, "null static potential");
  if (v_kind == GPE_V_CPLX128 && p->kind == GPE_IMAGINARY)
    return fail(GPE_ERR_ARG, "imaginary time takes a real (float64) static potential");
  return build_static(p, v, v_kind, (cudaStream_t)stream);
}

int gpe_step(gpe_plan* p, void* psi, int nsteps, long long step0, void* stream) {
  if (!p || !psi) return fail(GPE_ERR_ARG, "null argument");
  if (nsteps < 0) return fail(GPE_ERR_ARG, "nsteps must be >= 0");
  cudaStream_t st = (cudaStream_t)stream;
  const bool imag = p->kind == GPE_IMAGINARY;
  PdlChain chain(p);
  if (p->plane && nsteps > 0) {
    // per step: XKIN, then one plane-fused launch [inverse y, z, forward y]; the
    // first call opens with [Z1, forward y], the last step ends with [inverse y, Z2]
    const FastOps yf = mk_ops(FM_PLAIN), yi = mk_ops(FM_PLAIN, 1);
    {
      const FastOps ops[2] = {mk_ops(FM_Z1), yf};
      TRY(psweep(p, psi, FM_Z1, ops, 2, 0, t_mid_host(p, step0), 0.0, st));
    }
    for (int s = 0; s < nsteps; ++s) {
      const double t = t_mid_host(p, step0 + s), tn = t_mid_host(p, step0 + s + 1);
      Sweep x = mk_sweep(psi, psi);
      TRY(fsweep(p, AX_X, x, mk_ops(FM_XKIN), st));
      const bool more = s + 1 < nsteps;
      if (more && !imag) {
        const FastOps ops[3] = {yi, mk_ops(FM_Z21), yf};
        TRY(psweep(p, psi, FM_Z21, ops, 3, 1, t, tn, st));
        continue;
      }
      const FastOps ops[2] = {yi, mk_ops(FM_Z2, 0, 0, 0, imag ? 1 : 0)};
      TRY(psweep(p, psi, FM_Z2, ops, 2, 1, t, 0.0, st));
      if (more) {
        const FastOps ops2[2] = {mk_ops(FM_Z1, 0, 0, 1), yf};
        TRY(psweep(p, psi, FM_Z1, ops2, 2, 0, tn, 0.0, st));
      }
    }
    if (imag) TRY(scale_sweep(p, psi, st));
    return GPE_OK;
  }
  if (p->fast && nsteps > 0) {
    // real time fuses each step's last z sweep with the next step's first
    TRY(fast_front(p, psi, t_mid_host(p, step0), false, st));
    for (int s = 0; s < nsteps; ++s) {
      const double t = t_mid_host(p, step0 + s);
      TRY(fast_middle(p, psi, st));
      const bool fuse = !imag && s + 1 < nsteps;
      TRY(fast_back(p, psi, t, t_mid_host(p, step0 + s + 1), fuse, st));
      if (imag && s + 1 < nsteps) TRY(fast_front(p, psi, t_mid_host(p, step0 + s + 1), true, st));
    }
    if (imag) TRY(scale_sweep(p, psi, st));
    return GPE_OK;
  }
  for (int s = 0; s < nsteps; ++s) TRY(strang_step(p, psi, t_mid_host(p, step0 + s), imag && s > 0, st));
  if (imag && nsteps > 0) TRY(scale_sweep(p, psi, st));
  return GPE_OK;
}

int gpe_step_at(gpe_plan* p, void* psi, double t, void* stream) {
  if (!p || !psi) return fail(GPE_ERR_ARG, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  // reference: t_mid = float(t) + dt/2 (gpe/make_propagator.py:94)
  const double tm = t + p->dt / 2;
  PdlChain chain(p);
  if (p->fast) {
    TRY(fast_front(p, psi, tm, false, st));
    TRY(fast_middle(p, psi, st));
    TRY(fast_back(p, psi, tm, tm, false, st));
  } else {
    TRY(strang_step(p, psi, tm, false, st));
  }
  if (p->kind == GPE_IMAGINARY) TRY(scale_sweep(p, psi, st));
  return GPE_OK;
}

int gpe_halfstep(gpe_plan* p, void* psi, double t, void* stream) {
  if (!p || !psi) return fail(GPE_ERR_ARG, "null argument");
  Sweep s = mk_sweep(psi, psi);
  s.pre = PW_HALF1;
  s.t1 = t;
  return sweep(p, AX_Z, s, (cudaStream_t)stream);
}

int gpe_fft3d(gpe_plan* p, const void* in, void* out, int inverse, void* stream) {
  if (!p || !in || !out) return fail(GPE_ERR_ARG, "null argument");
  return fft3d(p, in, out, inverse != 0, (cudaStream_t)stream);
}

int gpe_normalise(gpe_plan* p, void* psi, void* stream) {
  if (!p || !psi) return fail(GPE_ERR_ARG, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  TRY(norm_sweep(p, psi, st));
  return scale_sweep(p, psi, st);
}

int gpe_norm(gpe_plan* p, const void* psi, double* norm, void* stream) {
  if (!p || !psi || !norm) return fail(GPE_ERR_ARG, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  TRY(norm_sweep(p, psi, st));
  CU(cudaMemcpyAsync(norm, p->d_scale + 2, sizeof(double), cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  return GPE_OK;
}

int gpe_kinetic_energy(gpe_plan* p, const void* psi_k, double* e_kin, void* stream) {
  if (!p || !psi_k || !e_kin) return fail(GPE_ERR_ARG, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  int nb = 0;
  TRY(kspace_reduce(p, psi_k, false, nb, st));
  std::vector<double> h;
  TRY(finish_diag(p, 0, nb, false, h, st));
  *e_kin = h[3] * p->ph.dx3 * p->ph.inv_m;
  return GPE_OK;
}

int gpe_nk_extraction(gpe_plan* p, const void* psi_k, double* occupation, long long* counts, void* stream) {
  if (!p || !psi_k) return fail(GPE_ERR_ARG, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  int nb = 0;
  TRY(kspace_reduce(p, psi_k, true, nb, st));
  std::vector<double> h;
  TRY(finish_diag(p, 0, nb, true, h, st));
  const double f = p->ph.dx3 * p->ph.inv_m;
  if (occupation)
    for (int b = 0; b < p->nbins; ++b) occupation[b] = h[4 + b] * f;
  if (counts)
    for (int b = 0; b < p->nbins; ++b) counts[b] = p->counts[b];
  return GPE_OK;
}

int gpe_diagnostics(gpe_plan* p, const void* psi, double t, double* scalars, double* nk, long long* counts,
                    void* stream) {
  if (!p || !psi || !scalars) return fail(GPE_ERR_ARG, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  TRY(ensure_work(p));
  TRY(ensure_hist(p));
  const bool hist = nk != nullptr;
  TRY(diag_launch(p, psi, t, hist, st));
  int na = 0, nb = 0;
  diag_tiles(p, diag_fast(p, hist), na, nb);
  std::vector<double> h;
  TRY(finish_diag(p, na, nb, hist, h, st));
  diag_scalars(p, h.data(), scalars);
  if (nk)
    for (int b = 0; b < p->nbins; ++b) nk[b] = h[4 + b] * p->ph.dx3 * p->ph.inv_m;
  if (counts)
    for (int b = 0; b < p->nbins; ++b) counts[b] = p->counts[b];
  return GPE_OK;
}

int gpe_launch_count(const gpe_plan* p, long long* count) {
  if (!p || !count) return fail(GPE_ERR_ARG, "null argument");
  *count = p->launches;
  return GPE_OK;
}

int gpe_profile(gpe_plan* p, int enable) {
  if (!p) return fail(GPE_ERR_ARG, "null plan");
  CU(cudaDeviceSynchronize());
  for (auto& r : p->recs) { p->pool.push_back(r.a); p->pool.push_back(r.b); }
  p->recs.clear();
  p->prof = enable != 0;
  return GPE_OK;
}

int gpe_profile_read(gpe_plan* p, double* ms, long long* count) {
  if (!p || !ms || !count) return fail(GPE_ERR_ARG, "null argument");
  for (int a = 0; a < 3; ++a) { ms[a] = 0.0; count[a] = 0; }
  for (auto& r : p->recs) {
    CU(cudaEventSynchronize(r.b));
    float t = 0.f;
    CU(cudaEventElapsedTime(&t, r.a, r.b));
    ms[r.ax] += t;
    count[r.ax] += 1;
  }
  return GPE_OK;
}

int gpe_projections(gpe_plan* p, const void* psi, unsigned which, double* out, void* stream) {
  if (!p || !psi || (which && !out)) return fail(GPE_ERR_ARG, "null argument");
  if (which >> 7) return fail(GPE_ERR_ARG, "unknown projection bits");
  cudaStream_t st = (cudaStream_t)stream;
  return p->dtype == GPE_C64 ? projections<float>(p, psi, which, out, st)
                             : projections<double>(p, psi, which, out, st);
}

int gpe_angular_momentum(gpe_plan* p, const void* psi, double* lz, void* stream) {
  if (!p || !psi || !lz) return fail(GPE_ERR_ARG, "null argument");
  return angular_momentum(p, psi, lz, (cudaStream_t)stream);
}

int gpe_status(gpe_plan* p, int* flags, void* stream) {
  if (!p || !flags) return fail(GPE_ERR_ARG, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  CU(cudaMemcpyAsync(flags, p->d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
  CU(cudaMemsetAsync(p->d_status, 0, sizeof(int), st));
  CU(cudaStreamSynchronize(st));
  return GPE_OK;
}

}  // extern "C"

// ================================================================ batches
// Many independent imaginary-time solves of mixed grid sizes advanced together.
// Instances are grouped by grid size; every sweep of a step is one launch per
// group whose grid is (tiles, instances): blockIdx.y picks the instance, whose
// physics and pointers come from device arrays.  One Strang step of all groups
// is captured once as a CUDA graph with one parallel branch per group and
// replayed for every further step.
struct gpe_batch {
  int dtype = 0;
  std::vector<gpe_plan*> plans;
  struct Group {
    int n = 0;
    int kind = GPE_IMAGINARY;   // real-time groups: no renormalisation, per-step clock
    bool fast = false;
    std::vector<int> all;       // every instance of this size
    std::vector<int> members;   // the bound (active) ones
    Phys* d_ph = nullptr;
    Sweep* d_sw = nullptr;      // [roles][members]
    int cap = 0;
    cudaStream_t stream = nullptr;
    int priority = 0;           // of `stream`: that of the stream the batch was last bound on
    cudaEvent_t ev = nullptr;
    int uploaded = 0;           // member count the device arrays hold
    // real time: half-step time and beam centres of every step of the current call,
    // [step][member][6] = {t_mid, cx, cy, t_end, cx, cy}, and each member's position in it
    double* d_times = nullptr;
    double* h_times = nullptr;  // pinned staging of the same
    int* d_tick = nullptr;
    int times_cap = 0;          // members the arrays hold (for BATCH_CLOCK_STEPS steps)
  };
  std::vector<Group> groups;
  std::vector<void*> psis;
  std::vector<long long> clock;   // real time: steps taken by each instance (t = clock * dt)
  cudaGraphExec_t graph = nullptr;
  cudaGraph_t graph_def = nullptr;
  cudaEvent_t fork = nullptr;
  cudaStream_t cap = nullptr;   // private stream the step graph is captured on
  cudaEvent_t ready = nullptr;
  double* h_sums = nullptr;     // pinned, 4 doubles per instance
  long long launches = 0;
  std::vector<gpe_plan*> parked;  // removed instances awaiting a bulk free
  DiagJob* d_jobs = nullptr;      // finish jobs of the bound instances
  double* d_sums = nullptr;       // 4 doubles per instance
  int jobs = 0, jobs_cap = 0, sums_cap = 0;
  // on-device convergence (gpe_batch_run): per-instance live flag (read by every
  // batched launch of an imaginary-time instance; 1 outside gpe_batch_run), steps
  // and last energy, with pinned staging for the caller's copies
  int* d_live = nullptr;
  long long* d_steps = nullptr;
  double* d_elast = nullptr;
  void* h_run = nullptr;
  int live_cap = 0;
};

namespace {

enum { ROLE_Z1N = 0, ROLE_Z1, ROLE_Y1, ROLE_X, ROLE_Y2, ROLE_Z2, ROLE_SC, ROLE_DZ, ROLE_DY, ROLE_DX, ROLE_COUNT };

// steps of a real-time group's time table per upload (longer calls are chunked)
constexpr int BATCH_CLOCK_STEPS = 1024;

// Group of (grid size, kind), created on first use.
int batch_group(gpe_batch* b, const gpe_plan* p, bool make_streams) {
  for (size_t q = 0; q < b->groups.size(); ++q)
    if (b->groups[q].n == p->n && b->groups[q].kind == p->kind) return (int)q;
  gpe_batch::Group g;
  g.n = p->n;
  g.kind = p->kind;
  g.fast = p->fast;
  if (make_streams) {
    if (cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking) != cudaSuccess) return -1;
    if (cudaEventCreateWithFlags(&g.ev, cudaEventDisableTiming) != cudaSuccess) return -1;
  }
  b->groups.push_back(g);
  return (int)b->groups.size() - 1;
}

// What a batch instance may be: imaginary time, or real time with the built-in
// stirring beam (dynamic expressions need the per-launch line table of a plan).
int batch_check_desc(const gpe_batch* b, const gpe_desc* d) {
  if (d->kind != GPE_IMAGINARY && d->kind != GPE_REAL) return fail(GPE_ERR_ARG, "kind must be imaginary or real");
  if (d->kind == GPE_REAL && d->dynamic_g_len)
    return fail(GPE_ERR_ARG, "batched real-time instances take the built-in beam, not dynamic expressions");
  if (d->dtype != b->dtype) return fail(GPE_ERR_ARG, "all instances of a batch share one dtype");
  return GPE_OK;
}

// Fill and upload the time tables of every bound real-time group for steps
// [first, first + count) of the call (count <= BATCH_CLOCK_STEPS).
int batch_times(gpe_batch* b, long long first, int count, cudaStream_t st) {
  for (auto& g : b->groups) {
    if (g.kind != GPE_REAL || g.members.empty()) continue;
    const int m = (int)g.members.size();
    for (int q = 0; q < m; ++q) {
      const gpe_plan* p = b->plans[g.members[q]];
      const long long s0 = b->clock[g.members[q]] + first;
      for (int k = 0; k < count; ++k) {
        Sweep a;
        a.t1 = t_mid_host(p, s0 + k);              // gpe/launch.py:10 + gpe/make_propagator.py:94
        a.t2 = (double)(s0 + k + 1) * p->dt;       // the state's time after the step
        beam_centres(p, a);
        double* e = g.h_times + ((size_t)k * m + q) * 6;
        e[0] = a.t1; e[1] = a.bc1x; e[2] = a.bc1y;
        e[3] = a.t2; e[4] = a.bc2x; e[5] = a.bc2y;
      }
    }
    CU(cudaMemcpyAsync(g.d_times, g.h_times, sizeof(double) * 6 * (size_t)m * count, cudaMemcpyHostToDevice, st));
    CU(cudaMemsetAsync(g.d_tick, 0, sizeof(int) * m, st));
  }
  return GPE_OK;
}

void batch_free_graph(gpe_batch* b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  if (b->graph_def) cudaGraphDestroy(b->graph_def);
  b->graph = nullptr;
  b->graph_def = nullptr;
}

void batch_free(gpe_batch* b) {
  batch_free_graph(b);
  for (auto& g : b->groups) {
    if (g.d_ph) cudaFree(g.d_ph);
    if (g.d_sw) cudaFree(g.d_sw);
    if (g.d_times) cudaFree(g.d_times);
    if (g.d_tick) cudaFree(g.d_tick);
    if (g.h_times) cudaFreeHost(g.h_times);
    if (g.stream) cudaStreamDestroy(g.stream);
    if (g.ev) cudaEventDestroy(g.ev);
  }
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->ready) cudaEventDestroy(b->ready);
  if (b->cap) cudaStreamDestroy(b->cap);
  if (b->h_sums) cudaFreeHost(b->h_sums);
  if (b->d_jobs) cudaFree(b->d_jobs);
  if (b->d_sums) cudaFree(b->d_sums);
  if (b->d_live) cudaFree(b->d_live);
  if (b->d_steps) cudaFree(b->d_steps);
  if (b->d_elast) cudaFree(b->d_elast);
  if (b->h_run) cudaFreeHost(b->h_run);
  for (auto* p : b->plans)
    if (p) free_plan(p);
  for (auto* p : b->parked) free_plan(p);
  delete b;
}

Sweep role_sweep(int role, void* psi, gpe_plan* p) {
  Sweep s = mk_sweep(psi, psi);
  s.partial = p->d_partial;
  s.t1 = s.t2 = p->dt / 2;
  switch (role) {
    case ROLE_Z1N: s.pre = PW_HALF1; s.fft1 = 1; break;
    case ROLE_Z1: s.pre = PW_HALF1 | PW_SCALE; s.fft1 = 1; break;
    case ROLE_Y1: s.fft1 = 1; break;
    case ROLE_X: s.fft1 = 1; s.mid = PW_KIN | PW_CONJ_LAST; s.fft2 = 1; s.post = PW_CONJ_FIRST; break;
    case ROLE_Y2: s.pre = PW_CONJ_LAST; s.fft1 = 1; s.post = PW_CONJ_FIRST; break;
    case ROLE_Z2:
      s.pre = PW_CONJ_LAST;
      s.fft1 = 1;
      s.post = PW_CONJ_FIRST | PW_INVM | PW_HALF1 | (p->kind == GPE_IMAGINARY ? PW_NORM : 0u);
      break;
    case ROLE_SC: s.pre = PW_SCALE; break;
    // diagnostics: real-space sums + forward z/y into the work buffer, k-space sums in x
    case ROLE_DZ: s.dst = p->d_work; s.pre = PW_DIAG_R; s.fft1 = 1; s.t1 = 0.0; break;
    case ROLE_DY: s.src = p->d_work; s.dst = p->d_work; s.fft1 = 1; break;
    default:
      // (the register-resident x sweep skips the shell histogram: batches finish energies only)
      s.src = p->d_work; s.dst = nullptr; s.fft1 = 1; s.post = PW_DIAG_K;
      s.partial = p->d_partial + 4 * (size_t)p->max_tiles; s.hist = diag_fast(p, false) ? nullptr : p->d_hist;
      break;
  }
  return s;
}

int role_axis(int role) {
  if (role == ROLE_Y1 || role == ROLE_Y2 || role == ROLE_DY) return AX_Y;
  if (role == ROLE_X || role == ROLE_DX) return AX_X;
  return AX_Z;
}

template <typename R>
int group_launch(gpe_batch* b, gpe_batch::Group& g, int role, cudaStream_t st) {
  const int count = (int)g.members.size();
  if (!count) return GPE_OK;
  if (g.uploaded != count) return fail(GPE_ERR_ARG, "batch membership changed without gpe_batch_bind");
  const Sweep* sws = g.d_sw + (size_t)role * count;
  const int ax = role_axis(role);
  if (role == ROLE_SC) {
    // lagged renormalisation: an elementwise pass per instance
    const long long elems = (long long)g.n * g.n * g.n;
    k_scale_batch<R><<<dim3((unsigned)((elems + 1023) / 1024), (unsigned)count), 256, 0, st>>>(sws, elems);
    CU(cudaGetLastError());
    ++b->launches;
    return GPE_OK;
  }
  if (g.fast) {
    FastOps op = mk_ops(FM_PLAIN);
    const int fax = ax == AX_Z ? FZ : ax == AX_Y ? FY : FX;
    switch (role) {
      case ROLE_Z1N: op = mk_ops(FM_Z1, 0, 0, 0); break;
      case ROLE_Z1: op = mk_ops(FM_Z1, 0, 0, 1); break;
      case ROLE_Y1: op = mk_ops(FM_PLAIN); break;
      case ROLE_X: op = mk_ops(FM_XKIN); break;
      case ROLE_Y2: op = mk_ops(FM_PLAIN, 1); break;
      case ROLE_DZ: op = mk_ops(FM_DIAGR); break;
      case ROLE_DY: op = mk_ops(FM_PLAIN); break;
      case ROLE_DX: op = mk_ops(FM_DIAGK); break;
      default: op = mk_ops(FM_Z2, 0, 0, 0, g.kind == GPE_IMAGINARY ? 1 : 0); break;
    }
    CU(launch_fast_batch<R>(g.n, fax, g.d_ph, sws, count, op, st));
  } else {
    gpe_plan* p = b->plans[g.members[0]];
    Sweep geo = mk_sweep(nullptr, nullptr);
    int tiles = 0, threads = 0;
    size_t smem = 0;
    TRY(sweep_geometry<R>(p, ax, geo, tiles, threads, smem));
    CU(launch_sweep_batch<R>(ax, p->gen, g.d_ph, sws, count, tiles, threads, smem, st));
  }
  ++b->launches;
  return GPE_OK;
}

int group_role(gpe_batch* b, gpe_batch::Group& g, int role, cudaStream_t st) {
  return b->dtype == GPE_C64 ? group_launch<float>(b, g, role, st) : group_launch<double>(b, g, role, st);
}

int group_step(gpe_batch* b, gpe_batch::Group& g, bool scaled, cudaStream_t st) {
  if (g.kind == GPE_REAL) {
    // this step's half-step time and beam centres into the z sweeps' (and the
    // diagnostics') sweep descriptors
    const int m = (int)g.members.size();
    k_batch_clock<<<(m + 127) / 128, 128, 0, st>>>(g.d_sw, m, g.d_times, g.d_tick, ROLE_Z1N, ROLE_Z2, ROLE_DZ);
    CU(cudaGetLastError());
    ++b->launches;
    TRY(group_role(b, g, ROLE_Z1N, st));
    TRY(group_role(b, g, ROLE_Y1, st));
    TRY(group_role(b, g, ROLE_X, st));
    TRY(group_role(b, g, ROLE_Y2, st));
    return group_role(b, g, ROLE_Z2, st);
  }
  TRY(group_role(b, g, scaled ? ROLE_Z1 : ROLE_Z1N, st));
  TRY(group_role(b, g, ROLE_Y1, st));
  TRY(group_role(b, g, ROLE_X, st));
  TRY(group_role(b, g, ROLE_Y2, st));
  return group_role(b, g, ROLE_Z2, st);
}

// Every group's step on its own stream, forked from and joined back into `st`.
int batch_step_all(gpe_batch* b, bool scaled, cudaStream_t st) {
  CU(cudaEventRecord(b->fork, st));
  for (auto& g : b->groups) {
    if (g.members.empty()) continue;
    CU(cudaStreamWaitEvent(g.stream, b->fork, 0));
    TRY(group_step(b, g, scaled, g.stream));
    CU(cudaEventRecord(g.ev, g.stream));
    CU(cudaStreamWaitEvent(st, g.ev, 0));
  }
  return GPE_OK;
}

// Upload the per-instance structs of a group's members (layout [role][member]);
// `uploaded` records the member count the device arrays were built for.
int group_upload(gpe_batch* b, gpe_batch::Group& g) {
  const int m = (int)g.members.size();
  g.uploaded = m;
  if (!m) return GPE_OK;
  if (m > g.cap) {
    if (g.d_ph) cudaFree(g.d_ph);
    if (g.d_sw) cudaFree(g.d_sw);
    g.d_ph = nullptr;
    g.d_sw = nullptr;
    CU(cudaMalloc(&g.d_ph, sizeof(Phys) * m));
    CU(cudaMalloc(&g.d_sw, sizeof(Sweep) * m * ROLE_COUNT));
    g.cap = m;
  }
  if (g.kind == GPE_REAL && m > g.times_cap) {
    if (g.d_times) cudaFree(g.d_times);
    if (g.d_tick) cudaFree(g.d_tick);
    if (g.h_times) cudaFreeHost(g.h_times);
    g.d_times = nullptr;
    g.d_tick = nullptr;
    g.h_times = nullptr;
    const size_t bytes = sizeof(double) * 6 * (size_t)m * BATCH_CLOCK_STEPS;
    CU(cudaMalloc(&g.d_times, bytes));
    CU(cudaMallocHost(&g.h_times, bytes));
    CU(cudaMalloc(&g.d_tick, sizeof(int) * m));
    g.times_cap = m;
  }
  std::vector<Phys> hph(m);
  std::vector<Sweep> hsw((size_t)m * ROLE_COUNT);
  for (int q = 0; q < m; ++q) {
    gpe_plan* p = b->plans[g.members[q]];
    TRY(ensure_work(p));
    TRY(ensure_hist(p));
    hph[q] = p->ph;
    for (int role = 0; role < ROLE_COUNT; ++role) {
      Sweep s = role_sweep(role, b->psis[g.members[q]], p);
      if (g.kind == GPE_IMAGINARY && b->d_live) s.live = b->d_live + g.members[q];
      if (g.kind == GPE_REAL && role == ROLE_DZ) {
        // diagnostics at the instance's current time (the clock kernel keeps it current)
        s.t1 = s.t2 = (double)b->clock[g.members[q]] * p->dt;
        beam_centres(p, s);
      }
      int tiles = 0, threads = 0;
      size_t smem = 0;
      const int rc = b->dtype == GPE_C64 ? sweep_geometry<float>(p, role_axis(role), s, tiles, threads, smem)
                                         : sweep_geometry<double>(p, role_axis(role), s, tiles, threads, smem);
      if (rc != GPE_OK) return rc;
      hsw[(size_t)role * m + q] = s;
    }
  }
  CU(cudaMemcpyAsync(g.d_ph, hph.data(), sizeof(Phys) * m, cudaMemcpyHostToDevice, g.stream));
  CU(cudaMemcpyAsync(g.d_sw, hsw.data(), sizeof(Sweep) * m * ROLE_COUNT, cudaMemcpyHostToDevice, g.stream));
  CU(cudaStreamSynchronize(g.stream));
  return GPE_OK;
}

// Finish jobs (one per bound instance) and the device sums array.
int jobs_upload(gpe_batch* b) {
  std::vector<DiagJob> jobs;
  for (auto& g : b->groups)
    for (int i : g.members) {
      const gpe_plan* p = b->plans[i];
      DiagJob j;
      j.pa = p->d_partial;
      j.pb = p->d_partial + 4 * (size_t)p->max_tiles;
      diag_tiles(p, diag_fast(p, false), j.na, j.nb);
      j.index = i;
      j.imag = p->kind == GPE_IMAGINARY;
      j.ckin = p->ckin;
      j.dx3 = p->ph.dx3;
      j.inv_m = p->ph.inv_m;
      j.beta = p->beta;
      jobs.push_back(j);
    }
  b->jobs = (int)jobs.size();
  if (b->jobs > b->jobs_cap) {
    if (b->d_jobs) cudaFree(b->d_jobs);
    b->d_jobs = nullptr;
    CU(cudaMalloc(&b->d_jobs, sizeof(DiagJob) * b->jobs));
    b->jobs_cap = b->jobs;
  }
  const int n = (int)b->plans.size();
  if (n > b->sums_cap) {
    if (b->d_sums) cudaFree(b->d_sums);
    b->d_sums = nullptr;
    CU(cudaMalloc(&b->d_sums, sizeof(double) * 4 * n));
    b->sums_cap = n;
  }
  if (b->jobs) {
    CU(cudaMemcpyAsync(b->d_jobs, jobs.data(), sizeof(DiagJob) * b->jobs, cudaMemcpyHostToDevice, b->cap));
    CU(cudaStreamSynchronize(b->cap));
  }
  return GPE_OK;
}

// Live flags (and the run state arrays) for `count` slots, every flag 1.  The
// arrays move only here, before the groups' descriptors are rebuilt by the bind.
int live_reset(gpe_batch* b, int count) {
  if (count > b->live_cap) {
    const int cap = std::max(count, 2 * b->live_cap);
    if (b->d_live) cudaFree(b->d_live);
    if (b->d_steps) cudaFree(b->d_steps);
    if (b->d_elast) cudaFree(b->d_elast);
    if (b->h_run) cudaFreeHost(b->h_run);
    b->d_live = nullptr;
    b->d_steps = nullptr;
    b->d_elast = nullptr;
    b->h_run = nullptr;
    b->live_cap = 0;
    CU(cudaMalloc(&b->d_live, sizeof(int) * cap));
    CU(cudaMalloc(&b->d_steps, sizeof(long long) * cap));
    CU(cudaMalloc(&b->d_elast, sizeof(double) * cap));
    CU(cudaMallocHost(&b->h_run, (sizeof(int) + sizeof(long long) + sizeof(double) + 4 * sizeof(double)) * cap));
    b->live_cap = cap;
  }
  if (count > 0) {
    k_fill_int<<<(count + 255) / 256, 256, 0, b->cap>>>(b->d_live, count, 1);
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(b->cap));
  }
  return GPE_OK;
}

}  // namespace

extern "C" {

int gpe_batch_create(const gpe_desc* descs, int count, gpe_batch** out) {
  if (!out || count < 0 || (count > 0 && !descs)) return fail(GPE_ERR_ARG, "descs (count >= 0) and out are required");
  *out = nullptr;
  gpe_batch* b = new gpe_batch();
  b->dtype = count > 0 ? descs[0].dtype : GPE_C64;
  for (int i = 0; i < count; ++i) {
    int rc = batch_check_desc(b, &descs[i]);
    if (rc != GPE_OK) { batch_free(b); return rc; }
    gpe_plan* p = nullptr;
    rc = create(&descs[i], &p);
    if (rc != GPE_OK) { batch_free(b); return rc; }
    b->plans.push_back(p);
    b->groups[batch_group(b, p, false)].all.push_back(i);
  }
  b->clock.assign(count, 0);
  for (auto& g : b->groups) {
    CU(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking));
    CU(cudaEventCreateWithFlags(&g.ev, cudaEventDisableTiming));
  }
  CU(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
  CU(cudaEventCreateWithFlags(&b->ready, cudaEventDisableTiming));
  CU(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
  CU(cudaMallocHost(&b->h_sums, sizeof(double) * 4 * (count > 0 ? count : 1)));
  b->psis.assign(count, nullptr);
  *out = b;
  return GPE_OK;
}

int gpe_batch_add(gpe_batch* b, const gpe_desc* d, int* index) {
  if (!b || !d || !index) return fail(GPE_ERR_ARG, "null argument");
  TRY(batch_check_desc(b, d));
  gpe_plan* p = nullptr;
  TRY(create(d, &p));
  int slot = -1;
  for (size_t i = 0; i < b->plans.size(); ++i)
    if (!b->plans[i]) { slot = (int)i; break; }
  if (slot < 0) {
    slot = (int)b->plans.size();
    b->plans.push_back(nullptr);
    b->psis.push_back(nullptr);
    b->clock.push_back(0);
    double* h = nullptr;
    CU(cudaMallocHost(&h, sizeof(double) * 4 * b->plans.size()));
    if (b->h_sums) cudaFreeHost(b->h_sums);
    b->h_sums = h;
  }
  b->plans[slot] = p;
  b->psis[slot] = nullptr;
  b->clock[slot] = 0;
  const int gi = batch_group(b, p, true);
  if (gi < 0) return fail(GPE_ERR_CUDA, "stream or event creation failed");
  b->groups[gi].all.push_back(slot);
  *index = slot;
  return GPE_OK;
}

// Removal requires the batch's work to be finished: call it after a synchronising
// call on the batch's stream (gpe_batch_diagnostics) or a stream synchronise.
int gpe_batch_remove(gpe_batch* b, int index) {
  if (!b || index < 0 || index >= (int)b->plans.size() || !b->plans[index])
    return fail(GPE_ERR_ARG, "no such batch instance");
  // The caller has synchronised the batch's stream (the graph is idle).  Freeing
  // device memory would wait for every stream of the device, so removed plans are
  // parked and freed together once enough have accumulated.  An instance that is
  // not bound (a rebind left it out) leaves without rebuilding the device tables.
  bool bound = false;
  for (auto& g : b->groups)
    bound = bound || std::find(g.members.begin(), g.members.end(), index) != g.members.end();
  if (bound) {
    for (auto& g : b->groups) CU(cudaStreamSynchronize(g.stream));
    batch_free_graph(b);
  }
  b->psis[index] = nullptr;
  for (auto& g : b->groups) {
    g.all.erase(std::remove(g.all.begin(), g.all.end(), index), g.all.end());
    const size_t before = g.members.size();
    g.members.erase(std::remove(g.members.begin(), g.members.end(), index), g.members.end());
    if (g.members.size() != before) TRY(group_upload(b, g));
  }
  if (bound) TRY(jobs_upload(b));
  b->parked.push_back(b->plans[index]);
  if (b->parked.size() >= 64) {
    for (auto* q : b->parked) free_plan(q);
    b->parked.clear();
  }
  b->plans[index] = nullptr;
  b->psis[index] = nullptr;
  return GPE_OK;
}

int gpe_batch_destroy(gpe_batch* b) {
  if (!b) return GPE_OK;
  cudaDeviceSynchronize();
  batch_free(b);
  return GPE_OK;
}

int gpe_batch_bind(gpe_batch* b, void* const* psis, const int* active, void* stream) {
  if (!b || !psis) return fail(GPE_ERR_ARG, "null argument");
  const int count = (int)b->plans.size();
  CU(cudaStreamSynchronize((cudaStream_t)stream));
  for (auto& g : b->groups) CU(cudaStreamSynchronize(g.stream));
  batch_free_graph(b);
  // the groups' streams run at the priority of the caller's stream (a server can put
  // its batch ahead of long real-time segments on lower-priority streams)
  int priority = 0;
  CU(cudaStreamGetPriority((cudaStream_t)stream, &priority));
  for (auto& g : b->groups)
    if (g.priority != priority) {
      CU(cudaStreamDestroy(g.stream));
      CU(cudaStreamCreateWithPriority(&g.stream, cudaStreamNonBlocking, priority));
      g.priority = priority;
    }
  for (int i = 0; i < count; ++i) b->psis[i] = b->plans[i] ? psis[i] : nullptr;
  TRY(live_reset(b, count));
  for (auto& g : b->groups) {
    g.members.clear();
    for (int i : g.all)
      if ((!active || active[i]) && b->psis[i]) g.members.push_back(i);
    TRY(group_upload(b, g));
  }
  return jobs_upload(b);
}

int gpe_batch_step(gpe_batch* b, int nsteps, void* stream) {
  if (!b) return fail(GPE_ERR_ARG, "null batch");
  if (nsteps <= 0) return GPE_OK;
  cudaStream_t st = (cudaStream_t)stream;
  bool any = false;
  for (auto& g : b->groups) any = any || !g.members.empty();
  if (!any) return GPE_OK;
  if (nsteps > 1 && !b->graph) {
    // capture on the batch's own stream (the caller's may be the legacy default stream)
    CU(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
    const int rc = batch_step_all(b, true, b->cap);
    cudaGraph_t gdef = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->cap, &gdef);
    if (rc != GPE_OK) { if (gdef) cudaGraphDestroy(gdef); return rc; }
    CU(e);
    b->graph_def = gdef;
    CU(cudaGraphInstantiate(&b->graph, gdef, 0));
  }
  for (int c0 = 0; c0 < nsteps; c0 += BATCH_CLOCK_STEPS) {
    const int count = std::min(BATCH_CLOCK_STEPS, nsteps - c0);
    if (c0 > 0) CU(cudaStreamSynchronize(st));   // the previous table has left the staging buffer
    TRY(batch_times(b, c0, count, st));
    for (int s = 0; s < count; ++s) {
      if (c0 + s == 0) TRY(batch_step_all(b, false, st));  // first step: psi is normalised, no pending scale
      else CU(cudaGraphLaunch(b->graph, st));
    }
  }
  for (auto& g : b->groups)
    if (g.kind == GPE_REAL)
      for (int i : g.members) b->clock[i] += nsteps;
  // apply the last renormalisation (imaginary-time groups)
  CU(cudaEventRecord(b->fork, st));
  for (auto& g : b->groups) {
    if (g.members.empty() || g.kind != GPE_IMAGINARY) continue;
    CU(cudaStreamWaitEvent(g.stream, b->fork, 0));
    TRY(group_role(b, g, ROLE_SC, g.stream));
    CU(cudaEventRecord(g.ev, g.stream));
    CU(cudaStreamWaitEvent(st, g.ev, 0));
  }
  return GPE_OK;
}

int gpe_batch_diagnostics(gpe_batch* b, double* scalars, void* stream) {
  if (!b || !scalars) return fail(GPE_ERR_ARG, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  if (!b->jobs) return GPE_OK;
  CU(cudaEventRecord(b->fork, st));
  for (auto& g : b->groups) {
    if (g.members.empty()) continue;
    CU(cudaStreamWaitEvent(g.stream, b->fork, 0));
    TRY(group_role(b, g, ROLE_DZ, g.stream));
    TRY(group_role(b, g, ROLE_DY, g.stream));
    TRY(group_role(b, g, ROLE_DX, g.stream));
    CU(cudaEventRecord(g.ev, g.stream));
    CU(cudaStreamWaitEvent(st, g.ev, 0));
  }
  k_finish_diag_batch<<<b->jobs, 256, 0, st>>>(b->d_jobs, b->d_sums);
  CU(cudaGetLastError());
  ++b->launches;
  const int n = (int)b->plans.size();
  CU(cudaMemcpyAsync(b->h_sums, b->d_sums, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  for (auto& g : b->groups)
    for (int i : g.members) diag_scalars(b->plans[i], b->h_sums + 4 * i, scalars + 6 * i);
  return GPE_OK;
}

// Chunks of imaginary-time steps with the convergence test on the device: per
// chunk, every live bound instance takes `chunk` steps (the first without a
// pending scale, the rest through the step graph), its lagged renormalisation,
// the diagnostic sweeps and the finish, then k_batch_converge freezes the
// instances that converged.  One synchronisation per call; the per-chunk work
// is that of gpe_batch_step(chunk) + gpe_batch_diagnostics, so results are the
// same bit for bit as a host loop over those calls that stops each instance at
// its check.
int gpe_batch_run(gpe_batch* b, int chunk, int nchunks, double tol, long long max_steps, int* live,
                  long long* steps, double* e_last, double* scalars, void* stream) {
  if (!b || !live || !steps || !e_last || !scalars) return fail(GPE_ERR_ARG, "null argument");
  if (chunk <= 0 || nchunks <= 0 || max_steps <= 0) return fail(GPE_ERR_ARG, "chunk, nchunks and max_steps must be > 0");
  cudaStream_t st = (cudaStream_t)stream;
  const int n = (int)b->plans.size();
  bool any = false;
  for (auto& g : b->groups) {
    if (g.members.empty()) continue;
    if (g.kind != GPE_IMAGINARY)
      return fail(GPE_ERR_ARG, "gpe_batch_run advances imaginary-time instances only (use gpe_batch_step)");
    if (g.uploaded != (int)g.members.size())
      return fail(GPE_ERR_ARG, "batch membership changed without gpe_batch_bind");
    any = true;
  }
  if (!any || !b->jobs) return GPE_OK;
  if (n > b->live_cap) return fail(GPE_ERR_ARG, "batch instances added without gpe_batch_bind");
  // the caller's state of the slots into the device arrays (through pinned staging)
  int* h_live = (int*)b->h_run;
  long long* h_steps = (long long*)(h_live + b->live_cap);
  double* h_elast = (double*)(h_steps + b->live_cap);
  double* h_sums = h_elast + b->live_cap;
  for (int i = 0; i < n; ++i) {
    h_live[i] = live[i] ? 1 : 0;
    h_steps[i] = steps[i];
    h_elast[i] = e_last[i];
  }
  CU(cudaMemcpyAsync(b->d_live, h_live, sizeof(int) * n, cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(b->d_steps, h_steps, sizeof(long long) * n, cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(b->d_elast, h_elast, sizeof(double) * n, cudaMemcpyHostToDevice, st));
  if (chunk > 1 && !b->graph) {
    CU(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
    const int rc = batch_step_all(b, true, b->cap);
    cudaGraph_t gdef = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->cap, &gdef);
    if (rc != GPE_OK) { if (gdef) cudaGraphDestroy(gdef); return rc; }
    CU(e);
    b->graph_def = gdef;
    CU(cudaGraphInstantiate(&b->graph, gdef, 0));
  }
  for (int c = 0; c < nchunks; ++c) {
    TRY(batch_step_all(b, false, st));
    for (int s = 1; s < chunk; ++s) CU(cudaGraphLaunch(b->graph, st));
    CU(cudaEventRecord(b->fork, st));
    for (auto& g : b->groups) {
      if (g.members.empty()) continue;
      CU(cudaStreamWaitEvent(g.stream, b->fork, 0));
      TRY(group_role(b, g, ROLE_SC, g.stream));
      TRY(group_role(b, g, ROLE_DZ, g.stream));
      TRY(group_role(b, g, ROLE_DY, g.stream));
      TRY(group_role(b, g, ROLE_DX, g.stream));
      CU(cudaEventRecord(g.ev, g.stream));
      CU(cudaStreamWaitEvent(st, g.ev, 0));
    }
    k_finish_diag_batch<<<b->jobs, 256, 0, st>>>(b->d_jobs, b->d_sums);
    CU(cudaGetLastError());
    k_batch_converge<<<(b->jobs + 127) / 128, 128, 0, st>>>(b->d_jobs, b->jobs, b->d_sums, chunk, tol, max_steps,
                                                            b->d_live, b->d_steps, b->d_elast);
    CU(cudaGetLastError());
    b->launches += 2;
  }
  CU(cudaMemcpyAsync(h_live, b->d_live, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
  CU(cudaMemcpyAsync(h_steps, b->d_steps, sizeof(long long) * n, cudaMemcpyDeviceToHost, st));
  CU(cudaMemcpyAsync(h_elast, b->d_elast, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  CU(cudaMemcpyAsync(h_sums, b->d_sums, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost, st));
  // every flag back to 1 (gpe_batch_step advances every bound instance)
  k_fill_int<<<(n + 255) / 256, 256, 0, st>>>(b->d_live, n, 1);
  CU(cudaGetLastError());
  ++b->launches;
  CU(cudaStreamSynchronize(st));
  for (auto& g : b->groups)
    for (int i : g.members) {
      live[i] = h_live[i];
      steps[i] = h_steps[i];
      e_last[i] = h_elast[i];
      diag_scalars(b->plans[i], h_sums + 4 * i, scalars + 6 * i);
    }
  return GPE_OK;
}

int gpe_batch_set_step(gpe_batch* b, int index, long long step) {
  if (!b || index < 0 || index >= (int)b->plans.size() || !b->plans[index])
    return fail(GPE_ERR_ARG, "no such batch instance");
  if (b->plans[index]->kind != GPE_REAL) return fail(GPE_ERR_ARG, "only real-time instances have a clock");
  if (step < 0) return fail(GPE_ERR_ARG, "step must be >= 0");
  for (auto& g : b->groups) CU(cudaStreamSynchronize(g.stream));
  b->clock[index] = step;
  for (auto& g : b->groups)
    if (std::find(g.members.begin(), g.members.end(), index) != g.members.end()) {
      batch_free_graph(b);
      TRY(group_upload(b, g));
    }
  return GPE_OK;
}

int gpe_batch_get_step(const gpe_batch* b, int index, long long* step) {
  if (!b || !step || index < 0 || index >= (int)b->plans.size() || !b->plans[index])
    return fail(GPE_ERR_ARG, "no such batch instance");
  *step = b->clock[index];
  return GPE_OK;
}

int gpe_batch_launch_count(const gpe_batch* b, long long* count) {
  if (!b || !count) return fail(GPE_ERR_ARG, "null argument");
  *count = b->launches;
  return GPE_OK;
}

}  // extern "C"
