"""Drop-in propagator factories (``gpe/make_propagator.py``).

``make_real_propagator(stage)`` / ``make_imag_propagator(stage)`` return the
per-step closure the reference returns: ``f(stage) -> psi`` for static
potentials, ``f(stage, t) -> psi`` when a time-dependent potential (or the
built-in stirring beam) is active.  The closure reads ``stage.psi``,
``stage.staticV``, ``stage.beta``, ``stage.k_array``, ``stage.x_array``,
``stage.dt`` and ``stage.N_grids`` at every call, validates them as the
reference does (AssertionError), and advances ``stage.psi`` in place with the
fused CUDA sweeps; the returned tensor is ``stage.psi`` itself.

Extensions read from the stage when present: ``kinetic_coeff`` (default 1.0,
the reference convention), ``beam`` (a :class:`Beam`) and ``nk_bins``.
complex64 ``psi`` runs the complex64 kernels (FP64 kept for reductions, the
renormalisation scale, kinetic factors and the beam angle).

Each closure also has ``closure.run(stage, nsteps, step0)``: ``nsteps`` steps
in one C-ABI call with ``t = i*dt`` for step ``i`` (``gpe/launch.py:8-13``).

The stage's arrays may be torch tensors or any CUDA array that exports DLPack
(the reference's CuPy arrays): they are viewed zero-copy, psi is advanced in
place, and the closure returns the caller's own ``stage.psi`` object.  Both
libraries enqueue on the legacy default stream unless told otherwise, so the
order against the caller's own work is kept.  A ``staticV`` that is not a torch
tensor is re-read when a different array (or buffer) is bound; the reference
never modifies it in place.
"""

import torch

from .expressions import from_cuda_text
from .plan import Plan


def _tensor(a):
    """Torch view of a CUDA array: a torch tensor as is, a DLPack producer (a
    CuPy array) zero-copy; anything else unchanged (rejected by the checks)."""
    if isinstance(a, torch.Tensor) or not hasattr(a, "__dlpack__"):
        return a
    return torch.utils.dlpack.from_dlpack(a)


class _Binding:
    """Plans of one propagator, keyed by what the reference reads per call."""

    def __init__(self, stage, kind):
        self.kind = kind
        pp = stage.potential_params
        self.static_expr = (from_cuda_text(str(pp["static"]["expression"]))
                            if pp["static"]["activate"] else "0")
        dyn = pp.get("dynamic", {"activate": False})
        self.dynamic_expr = (from_cuda_text(str(dyn["expression"]))
                             if kind == "real" and dyn["activate"] else "0")
        kc = getattr(stage, "k_cut_params", None) or {"activate": False}
        self.k_cut = float(kc["k_cut"]) if kind == "real" and kc["activate"] else None
        self.beam = getattr(stage, "beam", None) if kind == "real" else None
        self.ckin = float(getattr(stage, "kinetic_coeff", 1.0))
        self.nk_bins = int(getattr(stage, "nk_bins", 0) or 0)
        self.plans = {}
        self.static_seen = {}

    def check(self, stage):
        """The reference's per-call assertions (``gpe/make_propagator.py:20-36,66-81,117-133``);
        returns torch views of (psi, staticV, k_array, x_array)."""
        psi, V, k, x = (_tensor(a) for a in (stage.psi, stage.staticV, stage.k_array, stage.x_array))
        n = stage.N_grids
        assert isinstance(psi, torch.Tensor) and psi.is_cuda
        assert isinstance(V, torch.Tensor) and V.is_cuda
        assert psi.dtype in (torch.complex128, torch.complex64)
        if self.kind == "real":
            assert V.dtype == torch.complex128
        else:
            assert V.dtype == torch.float64
        assert psi.is_contiguous() and V.is_contiguous()
        assert tuple(psi.shape) == (n, n, n)
        assert V.shape == psi.shape
        assert isinstance(k, torch.Tensor) and k.dtype == torch.float64
        assert tuple(k.shape) == (n,) and k.is_contiguous()
        assert isinstance(x, torch.Tensor) and x.dtype == torch.float64
        assert tuple(x.shape) == (n,) and x.is_contiguous()
        return psi, V, k, x

    def plan(self, stage):
        """(plan, torch view of psi) for this call."""
        psi, V, k, x = self.check(stage)
        key = (psi.dtype, psi.device.index, int(stage.N_grids), float(stage.beta), float(stage.dt),
               id(stage.x_array), id(stage.k_array))
        plan = self.plans.get(key)
        if plan is None:
            with torch.cuda.device(psi.device):
                plan = Plan(stage.N_grids, x, k, dtype=psi.dtype,
                            kind=self.kind, beta=stage.beta, dt=stage.dt, kinetic_coeff=self.ckin,
                            static_expr=self.static_expr, dynamic_expr=self.dynamic_expr,
                            k_cut=self.k_cut, beam=self.beam, nk_bins=self.nk_bins)
            self.plans[key] = plan
        self.sync_static(plan, V, stage.staticV)
        return plan, psi

    def sync_static(self, plan, V, orig):
        """Re-read ``staticV`` only when it is a new array or (torch) was modified in place."""
        stamp = (id(orig), getattr(orig, "_version", 0), V.data_ptr())
        if self.static_seen.get(id(plan)) == stamp:
            return
        plan.set_static_potential(None if not bool(torch.any(V != 0)) else V)
        self.static_seen[id(plan)] = stamp

    @property
    def dynamic(self):
        return self.dynamic_expr != "0" or self.beam is not None


def make_real_propagator(stage):
    """``gpe/make_propagator.py:5-104``."""
    assert stage.type == "real"
    binding = _Binding(stage, "real")

    if not binding.dynamic:
        def time_independent_propagator(stage):
            plan, psi = binding.plan(stage)
            plan.step_at(psi, 0.0)
            return stage.psi
        fn = time_independent_propagator
    else:
        def time_dependent_propagator(stage, t):
            plan, psi = binding.plan(stage)
            plan.step_at(psi, float(t))
            return stage.psi
        fn = time_dependent_propagator

    def run(stage, nsteps, step0=0):
        plan, psi = binding.plan(stage)
        plan.step(psi, nsteps, step0)
        return stage.psi

    fn.run = run
    fn.binding = binding
    fn.dynamic = binding.dynamic
    return fn


def make_imag_propagator(stage):
    """``gpe/make_propagator.py:106-152``."""
    binding = _Binding(stage, "imaginary")

    def standard_imaginary_step(stage):
        plan, psi = binding.plan(stage)
        plan.step(psi, 1, 0)
        return stage.psi

    def run(stage, nsteps, step0=0):
        plan, psi = binding.plan(stage)
        plan.step(psi, nsteps, step0)
        return stage.psi

    standard_imaginary_step.run = run
    standard_imaginary_step.binding = binding
    standard_imaginary_step.dynamic = False
    return standard_imaginary_step


def make_real_spatial_kernel(stage):
    """Drop-in for ``gpe/make_kernel.py:4-84``: ``kernel(psi, t=0.0)`` applies the
    real-time local half-step at time ``t`` in place."""
    binding = _Binding(stage, "real")

    def kernel(psi, t=0.0):
        old = stage.psi
        stage.psi = psi
        try:
            plan, view = binding.plan(stage)
            plan.halfstep(view, t)
        finally:
            stage.psi = old
        return psi
    return kernel


def make_imag_spatial_kernel(stage):
    """Drop-in for ``gpe/make_kernel.py:86-120``."""
    binding = _Binding(stage, "imaginary")

    def kernel(psi, t=0.0):
        old = stage.psi
        stage.psi = psi
        try:
            plan, view = binding.plan(stage)
            plan.halfstep(view, t)
        finally:
            stage.psi = old
        return psi
    return kernel
