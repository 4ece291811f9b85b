"""Run the reference's own propagator code on the host CPU.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Works only where the
reference sources are present and ``GPE_REFERENCE`` names their root; it is
used to generate the golden fixtures in ``tests/golden`` and to pin the
``oracle.ssf`` restatement against the reference itself.

How: a NumPy-backed module is installed as ``cupy`` (the technique of the
reference's own CPU tests, ``tests/test_workflow.py:41-62``), but instead of
refusing to run kernels it executes them:

* ``RawKernel`` sources (``gpe/kernels.py``, ``gpe/make_kernel.py``,
  ``gpe/helper.py``) are compiled verbatim with ``g++`` against a tiny host
  ``cupy/complex.cuh`` (``std::complex``).  A launch runs every
  (block, thread) of the grid; kernels that call ``__syncthreads`` run each
  thread of a block as a coroutine on its own stack and switch at every
  barrier, so the shared-memory tree reductions of ``get_N`` execute as
  written.
* ``ElementwiseKernel`` / ``ReductionKernel`` bodies (``gpe/helper.py``,
  ``gpe/nk_extraction.py``) are compiled into broadcasting host loops.
* ``cp.fft`` is ``numpy.fft`` (pocketfft) in place of cuFFT.

Build products go to ``oracle/_ref/`` (git-ignored).
"""

import ctypes
import hashlib
import importlib
import os
from pathlib import Path
import re
import subprocess
import sys
from types import ModuleType, SimpleNamespace

import numpy as np

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
# The reference's source tree, from GPE_REFERENCE (no default): nothing on the
# product path, in the GPU tests or in the bench reads it.
REFERENCE = Path(os.environ["GPE_REFERENCE"]) if os.environ.get("GPE_REFERENCE") else None
UNSET = "GPE_REFERENCE is unset: set it to the reference's source tree to run the reference on the host"


def available():
    """True when GPE_REFERENCE names a tree holding the reference's sources."""
    return REFERENCE is not None and (REFERENCE / "gpe" / "make_propagator.py").exists()

_COMPLEX_HEADER = r"""
#pragma once
#include <complex>
#include <cmath>
#include <math.h>
using std::complex;
using std::exp;
using std::abs;
"""

# Single-threaded cooperative scheduler: one coroutine per CUDA thread of a block.
_RUNTIME = r"""
#include <cstdint>
#include <cstdlib>
#include <cstring>
struct uint3_ { unsigned x, y, z; };
static uint3_ threadIdx, blockIdx, blockDim, gridDim;
#define __global__
#define __device__
#define __forceinline__ inline
#define __shared__ static

extern "C" void gpe_ctx_swap(void** save_sp, void* load_sp);
__asm__(
  ".text\n.globl gpe_ctx_swap\n.type gpe_ctx_swap,@function\ngpe_ctx_swap:\n"
  "  pushq %rbp\n  pushq %rbx\n  pushq %r12\n  pushq %r13\n  pushq %r14\n  pushq %r15\n"
  "  movq %rsp, (%rdi)\n  movq %rsi, %rsp\n"
  "  popq %r15\n  popq %r14\n  popq %r13\n  popq %r12\n  popq %rbx\n  popq %rbp\n  ret\n");

static void* g_sched_sp;
static void** g_thread_sp;
static int* g_done;
static unsigned g_cur;
static void (*g_body)(void**);
static void** g_args;

static void __syncthreads() { gpe_ctx_swap(&g_thread_sp[g_cur], g_sched_sp); }

extern "C" void gpe_thread_entry() {
  g_body(g_args);
  g_done[g_cur] = 1;
  gpe_ctx_swap(&g_thread_sp[g_cur], g_sched_sp);
  abort();
}

static void run_grid(unsigned gx, unsigned bx, void (*body)(void**), void** args, int coop) {
  blockDim.x = bx; blockDim.y = blockDim.z = 1;
  gridDim.x = gx; gridDim.y = gridDim.z = 1;
  threadIdx.y = threadIdx.z = blockIdx.y = blockIdx.z = 0;
  if (!coop) {
    for (unsigned b = 0; b < gx; ++b) { blockIdx.x = b;
      for (unsigned t = 0; t < bx; ++t) { threadIdx.x = t; body(args); } }
    return;
  }
  const size_t stack = 64 * 1024;
  char* stacks = (char*)aligned_alloc(64, stack * bx);
  g_thread_sp = (void**)calloc(bx, sizeof(void*));
  g_done = (int*)calloc(bx, sizeof(int));
  g_body = body; g_args = args;
  for (unsigned b = 0; b < gx; ++b) {
    blockIdx.x = b;
    for (unsigned t = 0; t < bx; ++t) {
      uintptr_t top = ((uintptr_t)(stacks + (t + 1) * stack)) & ~(uintptr_t)15;
      void** sp = (void**)top;
      *--sp = 0;                              /* fake return address of the entry */
      *--sp = (void*)&gpe_thread_entry;       /* popped by ret */
      for (int r = 0; r < 6; ++r) *--sp = 0;  /* rbp rbx r12 r13 r14 r15 */
      g_thread_sp[t] = sp; g_done[t] = 0;
    }
    for (;;) {
      int live = 0;
      for (unsigned t = 0; t < bx; ++t) {
        if (g_done[t]) continue;
        live = 1; g_cur = t; threadIdx.x = t;
        gpe_ctx_swap(&g_sched_sp, g_thread_sp[t]);
      }
      if (!live) break;
    }
  }
  free(stacks); free(g_thread_sp); free(g_done);
}
"""

_CTYPES = {"complex128": "std::complex<double>", "complex64": "std::complex<float>",
           "float64": "double", "float32": "float", "int32": "int", "int64": "long long",
           "bool": "bool"}
_NP = {"complex128": np.complex128, "complex64": np.complex64, "float64": np.float64,
       "float32": np.float32, "int32": np.int32, "int64": np.int64, "bool": np.bool_}


def _compile(tag, source):
    OUT.mkdir(parents=True, exist_ok=True)
    inc = OUT / "include" / "cupy"
    inc.mkdir(parents=True, exist_ok=True)
    (inc / "complex.cuh").write_text(_COMPLEX_HEADER)
    digest = hashlib.sha256(source.encode()).hexdigest()[:16]
    cpp = OUT / f"{tag}_{digest}.cpp"
    so = OUT / f"{tag}_{digest}.so"
    if not so.exists():
        cpp.write_text(source)
        subprocess.run(["g++", "-O2", "-shared", "-fPIC", "-std=c++17",
                        "-I", str(OUT / "include"), str(cpp), "-o", str(so)],
                       check=True, capture_output=True)
    return ctypes.CDLL(str(so))


def _split_params(text):
    out, depth, cur = [], 0, ""
    for ch in text:
        if ch in "<(":
            depth += 1
        elif ch in ">)":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur.strip())
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur.strip())
    return out


class HostRawKernel:
    """``cupy.RawKernel`` executed on the host (see module docstring)."""

    def __init__(self, code, name, **kwargs):
        self.code, self.name = code, name
        self._lib = None

    def _build(self):
        m = re.search(r"\b" + re.escape(self.name) + r"\s*\(([^)]*)\)", self.code)
        params = _split_params(m.group(1))
        casts = []
        self.kinds = []
        for i, p in enumerate(params):
            ptype = re.sub(r"\s*\b\w+\s*$", "", p).replace("const", "").strip()
            if "*" in p:
                casts.append(f"({ptype})args[{i}]")
                self.kinds.append("ptr")
            else:
                casts.append(f"*({ptype}*)args[{i}]")
                self.kinds.append(ptype)
        coop = 1 if "__syncthreads" in self.code else 0
        src = (_RUNTIME + "\n" + self.code + "\n"
               f"static void body(void** args) {{ {self.name}({', '.join(casts)}); }}\n"
               'extern "C" void host_launch(unsigned gx, unsigned bx, void** args) '
               f"{{ run_grid(gx, bx, body, args, {coop}); }}\n")
        self._lib = _compile(self.name, src)
        self._lib.host_launch.argtypes = [ctypes.c_uint, ctypes.c_uint, ctypes.c_void_p]

    def __call__(self, grid, block, args, **kwargs):
        if self._lib is None:
            self._build()
        keep, ptrs = [], []
        for kind, a in zip(self.kinds, args):
            if kind == "ptr":
                assert isinstance(a, np.ndarray) and a.flags.c_contiguous
                ptrs.append(a.ctypes.data)
                continue
            if kind == "double":
                v = ctypes.c_double(float(a))
            elif kind == "float":
                v = ctypes.c_float(float(a))
            elif kind in ("long long", "long"):
                v = ctypes.c_longlong(int(a))
            elif kind == "int":
                v = ctypes.c_int(int(a))
            else:
                raise TypeError(f"unsupported kernel parameter type {kind}")
            keep.append(v)
            ptrs.append(ctypes.addressof(v))
        arr = (ctypes.c_void_p * len(ptrs))(*ptrs)
        self._lib.host_launch(int(grid[0]), int(block[0]), arr)


def _parse_decl(text):
    out = []
    for p in text.split(","):
        t, n = p.split()
        out.append((t, n))
    return out


class HostElementwiseKernel:
    """``cupy.ElementwiseKernel`` as a broadcasting host loop."""

    def __init__(self, in_params, out_params, operation, name, **kwargs):
        self.ins, self.outs = _parse_decl(in_params), _parse_decl(out_params)
        self.op, self.name = operation, name
        self._lib = None

    def _build(self):
        decl = ["long long n"]
        load = []
        for t, n in self.ins:
            decl.append(f"const {_CTYPES[t]}* {n}_p")
            load.append(f"{_CTYPES[t]} {n} = {n}_p[i];")
        for t, n in self.outs:
            decl.append(f"{_CTYPES[t]}* {n}_p")
            load.append(f"{_CTYPES[t]}& {n} = {n}_p[i];")
        src = (_COMPLEX_HEADER + "\nusing namespace std;\n"
               f'extern "C" void ew({", ".join(decl)}) {{\n'
               f"  for (long long i = 0; i < n; ++i) {{ {' '.join(load)}\n {self.op}\n }}\n}}\n")
        self._lib = _compile("ew_" + self.name, src)

    def __call__(self, *args):
        if self._lib is None:
            self._build()
        ins = [np.asarray(a) for a in args[:len(self.ins)]]
        outs = list(args[len(self.ins):])
        shape = np.broadcast_shapes(*[a.shape for a in ins], *[o.shape for o in outs])
        flat = [np.ascontiguousarray(np.broadcast_to(a.astype(_NP[t], copy=False), shape))
                for a, (t, _) in zip(ins, self.ins)]
        targets = [np.empty(shape, _NP[t]) for t, _ in self.outs]
        self._lib.ew(ctypes.c_longlong(int(np.prod(shape))),
                     *[ctypes.c_void_p(a.ctypes.data) for a in flat + targets])
        for o, tgt in zip(outs, targets):
            o[...] = tgt
        return outs


class HostReductionKernel:
    """``cupy.ReductionKernel`` (full reduction) as a sequential host loop."""

    def __init__(self, in_params, out_params, map_expr, reduce_expr, post_map_expr,
                 identity, name, reduce_type=None, **kwargs):
        self.ins, self.outs = _parse_decl(in_params), _parse_decl(out_params)
        self.map, self.red, self.post = map_expr, reduce_expr, post_map_expr
        self.identity, self.name = identity, name
        self.rtype = reduce_type or _CTYPES[self.outs[0][0]]
        self._lib = None

    def _build(self):
        decl = ["long long n"]
        load = []
        for t, n in self.ins:
            decl.append(f"const {_CTYPES[t]}* {n}_p")
            load.append(f"{_CTYPES[t]} {n} = {n}_p[i];")
        (ot, on), = self.outs
        decl.append(f"{_CTYPES[ot]}* {on}_p")
        src = (_COMPLEX_HEADER + "\nusing namespace std;\n"
               f'extern "C" void red({", ".join(decl)}) {{\n'
               f"  {self.rtype} a = ({self.rtype})({self.identity});\n"
               f"  for (long long i = 0; i < n; ++i) {{ {' '.join(load)}\n"
               f"    {self.rtype} b = ({self.map}); a = ({self.red}); }}\n"
               f"  {_CTYPES[ot]}& {on} = *{on}_p; {self.post};\n}}\n")
        self._lib = _compile("red_" + self.name, src)

    def __call__(self, *args, axis=None):
        if self._lib is None:
            self._build()
        ins = [np.asarray(a) for a in args[:len(self.ins)]]
        shape = np.broadcast_shapes(*[a.shape for a in ins])
        flat = [np.ascontiguousarray(np.broadcast_to(a.astype(_NP[t], copy=False), shape))
                for a, (t, _) in zip(ins, self.ins)]
        otype = _NP[self.outs[0][0]]
        if axis is None:
            out = np.zeros((), otype)
            self._lib.red(ctypes.c_longlong(int(np.prod(shape))),
                          *[ctypes.c_void_p(a.ctypes.data) for a in flat + [out]])
            return out
        # reduction along one axis: the same sequential loop over every line
        lines = [np.ascontiguousarray(np.moveaxis(a, axis, -1)) for a in flat]
        out = np.zeros(lines[0].shape[:-1], otype)
        cell = np.zeros((), otype)
        for idx in np.ndindex(out.shape):
            line = [np.ascontiguousarray(a[idx]) for a in lines]
            self._lib.red(ctypes.c_longlong(line[0].shape[0]),
                          *[ctypes.c_void_p(a.ctypes.data) for a in line + [cell]])
            out[idx] = cell
        return out


def install():
    """Install the shim as ``cupy`` and import the reference package ``gpe``."""
    if REFERENCE is None:
        raise RuntimeError(UNSET)
    if not available():
        raise RuntimeError(f"reference sources not found at {REFERENCE}")
    cupy = ModuleType("cupy")
    cupy.__getattr__ = lambda name: getattr(np, name)
    cupy.ndarray = np.ndarray
    cupy.asnumpy = np.asarray
    cupy.asarray = lambda a, dtype=None, blocking=False, **kw: np.array(a, dtype=dtype)
    cupy.asarray = lambda value, blocking=False, **kw: np.asarray(value, **kw)
    cupy.fft = SimpleNamespace(fftn=np.fft.fftn, ifftn=np.fft.ifftn, fftfreq=np.fft.fftfreq,
                               fftshift=np.fft.fftshift)
    cupy.RawKernel = HostRawKernel
    cupy.ElementwiseKernel = HostElementwiseKernel
    cupy.ReductionKernel = HostReductionKernel
    sys.modules["cupy"] = cupy
    if str(REFERENCE) not in sys.path:
        sys.path.insert(0, str(REFERENCE))
    mods = {name: importlib.import_module("gpe." + name)
            for name in ("make_propagator", "make_kernel", "kernels", "helper",
                         "nk_extraction", "grids", "initial_states", "expressions", "save", "state_io")}
    return SimpleNamespace(cp=cupy, **mods)


def reference_stage(ref, *, n, simulation_range, kind, beta, dt, static_expr="0",
                    dynamic_expr="0", k_cut=None, static_v=None):
    """The attributes of a reference ``stage`` (``gpe/stage.py:12-51``) that the
    propagator reads, built through the reference's own grid and expression code."""
    x, k = ref.grids.get_grids(n, simulation_range)
    static_on, dynamic_on = static_expr != "0", dynamic_expr != "0"
    potential = dict(
        static=dict(activate=static_on,
                    expression=ref.expressions.cuda_expression(static_expr)),
        dynamic=dict(activate=dynamic_on,
                     expression=ref.expressions.cuda_expression(dynamic_expr, time_dependent=True)))
    if static_v is None:
        static_v = (np.zeros((n,) * 3) if kind == "imaginary"
                    else np.zeros((n,) * 3, np.complex128))
    st = SimpleNamespace(
        type=kind, psi=None, staticV=np.ascontiguousarray(static_v), beta=float(beta),
        k_array=k, x_array=x, dt=float(dt), N_grids=n, potential_params=potential,
        k_cut_params=dict(activate=k_cut is not None, k_cut=k_cut or 0.0))
    if kind == "real":
        st.propagator = ref.make_propagator.make_real_propagator(st)
    else:
        st.propagator = ref.make_propagator.make_imag_propagator(st)
    return st


def run_reference(ref, st, psi, steps, step0=0):
    """``gpe/launch.py:8-13`` with outputs disabled."""
    st.psi = np.array(psi, dtype=np.complex128, order="C", copy=True)  # the step mutates its input
    dynamic = st.potential_params["dynamic"]["activate"]
    for i in range(step0, step0 + steps):
        st.psi = st.propagator(st, i * st.dt) if dynamic else st.propagator(st)
    return st.psi
