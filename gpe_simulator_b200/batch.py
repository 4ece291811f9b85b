"""Batched solves of mixed grid sizes: imaginary-time ground states and
real-time stirred evolutions.

Many independent solves (sweeps over g, trap aspect ratios, grid sizes and
stirring rates) advance together: ``gpe_batch_*`` groups the instances by grid
size and kind, launches every sweep once per group over (tiles x instances),
and replays one step of all groups from a CUDA graph with a parallel branch
per group.  Each instance runs exactly the arithmetic of its own single-plan
one-step call, so a solve gives the same bits alone and in the batch.
Real-time instances keep a clock (steps taken); each step evaluates the
stirring beam at ``t_mid = step * dt + dt/2`` as ``gpe/launch.py:10`` and
``gpe/make_propagator.py:94`` do.

:func:`solve` runs every instance until ``|E_k - E_{k-K}| / (K |E_k|) < tol``
(energy change per step, checked every ``K`` steps) or ``max_steps``, retiring
converged instances from the batch as it goes.
"""

import ctypes
from dataclasses import dataclass, field
import math

import numpy as np
import torch

from . import _lib
from .expressions import split_static
from .plan import _DTYPES, _dptr, _stream


@dataclass
class Instance:
    """One solve, in reference units (kinetic factor ``exp(-i c k^2 dt)``):
    ``kind`` ``"imaginary"`` (ground state) or ``"real"`` (stirred evolution with
    the built-in ``beam``, a :class:`~gpe_simulator_b200.plan.Beam`)."""
    n: int
    simulation_range: float
    beta: float
    dt: float
    static_expr: str = "0"
    kinetic_coeff: float = 1.0
    kind: str = "imaginary"
    beam: object = None
    x: np.ndarray = field(init=False, repr=False)
    k: np.ndarray = field(init=False, repr=False)

    def __post_init__(self):
        L = self.simulation_range
        self.x = np.linspace(-L / 2, L / 2, self.n, endpoint=False)
        self.k = 2 * np.pi * np.fft.fftfreq(self.n, L / self.n)


def _fill_desc(d, inst, dtype, keep):
    if inst.kind not in ("imaginary", "real"):
        raise KeyError("kind must be 'imaginary' or 'real'")
    d.n, d.dtype = inst.n, _DTYPES[dtype]
    d.kind = _lib.IMAGINARY if inst.kind == "imaginary" else _lib.REAL
    if inst.beam is not None:
        if inst.kind != "real":
            raise ValueError("Imaginary time evolution does not accept a time dependent potential.")
        b = inst.beam
        d.beam_enabled = 1
        d.beam_amp, d.beam_width, d.beam_radius, d.beam_omega, d.beam_t_ramp = (
            float(b.amp), float(b.width), float(b.radius), float(b.omega), float(b.t_ramp))
    d.beta, d.dt, d.kinetic_coeff = float(inst.beta), float(inst.dt), float(inst.kinetic_coeff)
    a, d.x_array = _dptr(inst.x)
    keep.append(a)
    a, d.k_array = _dptr(inst.k)
    keep.append(a)
    for name, prog in zip(("static_x", "static_y", "static_z", "static_g"), split_static(inst.static_expr)):
        if prog:
            a, ptr = _dptr(prog)
            keep.append(a)
            setattr(d, name, ptr)
            setattr(d, name + "_len", len(prog))


class Batch:
    def __init__(self, instances, dtype=torch.complex64):
        if not torch.cuda.is_available():
            raise RuntimeError("gpe_simulator_b200 needs a CUDA device (sm_100a)")
        self.lib = _lib.load()
        self.instances = list(instances)
        self.dtype = dtype
        count = len(self.instances)
        descs = (_lib.Desc * count)()
        self._keep = []
        for d, inst in zip(descs, self.instances):
            _fill_desc(d, inst, dtype, self._keep)
        handle = ctypes.c_void_p()
        _lib.check(self.lib.gpe_batch_create(ctypes.cast(descs, ctypes.c_void_p), count, ctypes.byref(handle)))
        self._h = handle
        self.psis = [None] * count
        self.active = np.ones(count, np.int32)

    def close(self):
        if getattr(self, "_h", None):
            torch.cuda.synchronize()
            self.lib.gpe_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, inst):
        """Add an instance to the running batch; returns its index (freed indices are reused)."""
        d = _lib.Desc()
        keep = []
        _fill_desc(d, inst, self.dtype, keep)
        idx = ctypes.c_int()
        _lib.check(self.lib.gpe_batch_add(self._h, ctypes.byref(d), ctypes.byref(idx)))
        i = idx.value
        if i == len(self.instances):
            self.instances.append(inst)
            self.psis.append(None)
            self.active = np.append(self.active, 0).astype(np.int32)
        else:
            self.instances[i] = inst
            self.psis[i] = None
            self.active[i] = 0
        return i

    def remove(self, index):
        """Drop instance ``index`` (its tensors stay with the caller)."""
        _lib.check(self.lib.gpe_batch_remove(self._h, int(index)))
        self.instances[index] = None
        self.psis[index] = None
        self.active[index] = 0

    def bind(self, psis, active=None):
        """Device states of every instance (C-contiguous cubes) and the active mask."""
        for i, (p, inst) in enumerate(zip(psis, self.instances)):
            if p is not None and inst is not None:
                if (not isinstance(p, torch.Tensor) or not p.is_cuda or p.dtype != self.dtype
                        or tuple(p.shape) != (inst.n,) * 3 or not p.is_contiguous()):
                    raise AssertionError(f"psi {i} must be a contiguous {self.dtype} CUDA cube of side {inst.n}")
        self.psis = list(psis)
        if active is None:
            # every instance that has a state is active
            active = [1 if (p is not None and inst is not None) else 0
                      for p, inst in zip(psis, self.instances)]
        self.active = np.asarray(active, np.int32).copy()
        ptrs = (ctypes.c_void_p * len(psis))(*[p.data_ptr() if p is not None else None for p in psis])
        act = self.active.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        _lib.check(self.lib.gpe_batch_bind(self._h, ptrs, act, _stream()))

    def step(self, nsteps):
        _lib.check(self.lib.gpe_batch_step(self._h, int(nsteps), _stream()))

    def diagnostics(self):
        """``(count, 6)`` array of N, E_kin, E_pot, E_int, E, mu (NaN for unbound instances)."""
        out = np.full((len(self.instances), 6), np.nan)
        _lib.check(self.lib.gpe_batch_diagnostics(
            self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), _stream()))
        return out

    def run(self, chunk, nchunks, tol, max_steps, live, steps, e_last):
        """Up to ``nchunks`` chunks of ``chunk`` imaginary-time steps with the
        convergence test on the device and one synchronisation (``gpe_batch_run``).
        ``live`` (int32), ``steps`` (int64) and ``e_last`` (float64), one entry per
        instance slot, are updated in place; returns the ``(count, 6)`` diagnostics
        at each bound instance's last check (NaN for unbound slots)."""
        n = len(self.instances)
        assert live.dtype == np.int32 and steps.dtype == np.int64 and e_last.dtype == np.float64
        assert live.shape == steps.shape == e_last.shape == (n,)
        assert live.flags.c_contiguous and steps.flags.c_contiguous and e_last.flags.c_contiguous
        out = np.full((n, 6), np.nan)
        dp = ctypes.POINTER(ctypes.c_double)
        _lib.check(self.lib.gpe_batch_run(
            self._h, int(chunk), int(nchunks), float(tol), int(max_steps), live.ctypes.data, steps.ctypes.data,
            e_last.ctypes.data_as(dp), out.ctypes.data_as(dp), _stream()))
        return out

    def set_step(self, index, step):
        """Clock of real-time instance ``index``: steps taken (its next step evaluates
        the beam at ``step * dt + dt/2``)."""
        _lib.check(self.lib.gpe_batch_set_step(self._h, int(index), int(step)))

    def get_step(self, index):
        out = ctypes.c_longlong()
        _lib.check(self.lib.gpe_batch_get_step(self._h, int(index), ctypes.byref(out)))
        return out.value

    def launch_count(self):
        out = ctypes.c_longlong()
        _lib.check(self.lib.gpe_batch_launch_count(self._h, ctypes.byref(out)))
        return out.value

    def solve(self, psis, tol=1e-9, max_steps=5000, check_every=10, checks_per_call=8):
        """Run every instance to ``|dE|/E < tol`` per step (checked every
        ``check_every`` steps) or ``max_steps`` (a multiple of ``check_every``).

        The checks run on the device (:meth:`run`), ``checks_per_call`` of them
        per synchronisation; converged instances stop at their check and leave
        the batch at the next rebind (when a quarter of the bound ones have
        stopped).  Returns ``(steps, energies)``: steps taken and final
        diagnostics per instance.
        """
        if max_steps % check_every:
            raise ValueError("max_steps must be a multiple of check_every")
        count = len(self.instances)
        self.bind(psis, np.ones(count, np.int32))
        steps = np.zeros(count, np.int64)
        e_last = self.diagnostics()[:, 4].copy()
        live = np.ones(count, np.int32)
        final = np.full((count, 6), np.nan)
        bound = count
        while live.any():
            was = live.copy()
            diag = self.run(check_every, checks_per_call, tol, max_steps, live, steps, e_last)
            stopped = (was == 1) & (live == 0)
            final[stopped] = diag[stopped]
            if live.any() and bound - int(live.sum()) >= max(1, bound // 4):
                self.bind(self.psis, live.copy())
                bound = int(live.sum())
        return steps, final


def solve_alone(inst, psi, dtype=torch.complex64, tol=1e-9, max_steps=5000, check_every=10):
    """One instance through a single plan with the convergence rule of
    :meth:`Batch.solve` (same checks, same step counts): the one-at-a-time
    baseline of a batched solve.  Returns ``(steps, diagnostics)``."""
    from .plan import Plan
    plan = Plan(inst.n, inst.x, inst.k, dtype=dtype, kind="imaginary", beta=inst.beta, dt=inst.dt,
                kinetic_coeff=inst.kinetic_coeff, static_expr=inst.static_expr)
    try:
        keys = ("N", "E_kin", "E_pot", "E_int", "E", "mu")
        d = plan.diagnostics(psi)
        last, steps = d["E"], 0
        while steps < max_steps:
            chunk = int(min(check_every, max_steps - steps))
            plan.step(psi, chunk)
            steps += chunk
            d = plan.diagnostics(psi)
            rate = abs(d["E"] - last) / (chunk * abs(d["E"])) if d["E"] != 0 else float("inf")
            last = d["E"]
            if rate < tol:
                break
        return steps, np.array([d[k] for k in keys])
    finally:
        plan.close()


def sweep_instances(count=64, seed=1, dt=1e-3):
    """The batched parameter sweep, in reference units.

    Grid side drawn from {48, 64, 96, 128, 160} with box [-L, L) for L in
    {6, 8, 10, 12, 14}; g log-uniform in [100, 5000]; lambda_y, lambda_z uniform
    in [0.5, 2]; V = (x^2 + lambda_y^2 y^2 + lambda_z^2 z^2)/2 and oscillator time
    step ``dt``.  Mapped exactly onto the reference convention: V x2, g x2, dt/2.
    """
    rng = np.random.default_rng(seed)
    sizes = [(48, 6.0), (64, 8.0), (96, 10.0), (128, 12.0), (160, 14.0)]
    out = []
    for _ in range(count):
        n, L = sizes[rng.integers(len(sizes))]
        g = float(math.exp(rng.uniform(math.log(100.0), math.log(5000.0))))
        ly, lz = rng.uniform(0.5, 2.0, 2)
        expr = f"x**2+{float(ly * ly)!r}*y**2+{float(lz * lz)!r}*z**2"
        out.append(Instance(n=n, simulation_range=2 * L, beta=2 * g, dt=dt / 2, static_expr=expr))
    return out


def stirring_instances(rates=(0.25, 0.5, 1.0), gs=(500.0, 1000.0), grids=((64, 16.0), (96, 20.0)),
                       dt=5e-4):
    """A stirring-rate sweep, in reference units: for every grid (side, box length),
    interaction g and final angular rate Omega of the beam (oscillator units A = 10,
    w = 0.5, R = 2, rate ramped 0 -> Omega over 200 steps), the trap
    V = (x^2 + 1.44 y^2 + 2.25 z^2)/2 with oscillator time step ``dt``.  Mapped
    exactly onto the reference convention: V x2, g x2, dt/2, rates x2."""
    from .plan import beam_in_reference_units
    out = []
    for n, L in grids:
        for g in gs:
            for omega in rates:
                beam = beam_in_reference_units(10.0, 0.5, 2.0, omega, 200 * dt)
                out.append(Instance(n=n, simulation_range=L, beta=2 * g, dt=dt / 2,
                                    static_expr="x**2+1.44*y**2+2.25*z**2", kind="real", beam=beam))
    return out


def initial_states(instances, dtype=torch.complex64, seed0=100, device="cuda"):
    """Seeded normalised Gaussian x (1 + 0.01 complex noise) for every instance."""
    out = []
    for i, inst in enumerate(instances):
        n, x = inst.n, inst.x
        rng = np.random.default_rng(seed0 + i)
        g = np.exp(-x ** 2 / 2)
        psi = g[:, None, None] * g[None, :, None] * g[None, None, :]
        psi = psi * (1 + 0.01 * (rng.standard_normal((n, n, n)) + 1j * rng.standard_normal((n, n, n))) / np.sqrt(2))
        psi /= np.sqrt(np.sum(np.abs(psi) ** 2) * (x[1] - x[0]) ** 3)
        out.append(torch.from_numpy(psi.astype(np.complex128)).to(device).to(dtype).contiguous())
    return out
