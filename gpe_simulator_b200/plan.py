"""``Plan``: one propagator configuration bound to the C ABI.

A plan owns the device tables of one grid/dtype/kind/potential combination
(twiddles, axis potentials, kinetic factors, reduction scratch) and launches
the fused sweeps on the current torch CUDA stream.  Tensors are torch CUDA
tensors, C-contiguous ``(N, N, N)`` complex64 or complex128.
"""

import ctypes
from dataclasses import dataclass
import math

import numpy as np
import torch

from . import _lib
from .expressions import compile_program, split_static


@dataclass
class Beam:
    """Rotating Gaussian stirring beam (plan units).

    ``V = amp * exp(-((x - radius cos th)^2 + (y - radius sin th)^2) / width^2)``,
    ``th(t) = omega (m^2 / (2 t_ramp) + t - m)``, ``m = min(t, t_ramp)``: the
    angular rate ramps linearly from 0 to ``omega`` over ``t_ramp``.  The angle
    is evaluated in FP64 on the device.
    """
    amp: float
    width: float
    radius: float
    omega: float
    t_ramp: float = 0.0

    def expression(self):
        """The same beam in the reference's potential grammar (``x, y, t``, ``abs``,
        ``cos``, ``sin``, ``exp``): ``min(t, t_ramp)`` written as
        ``(t + t_ramp - abs(t - t_ramp))/2``.  A plan given this as its dynamic
        expression runs the register-resident sweeps as with the built-in beam."""
        r = repr
        if self.t_ramp > 0:
            m = f"((t+{r(self.t_ramp)}-abs(t-{r(self.t_ramp)}))/2)"
            th = f"({r(self.omega)}*({m}**2/(2*{r(self.t_ramp)})+t-{m}))"
        else:
            th = f"({r(self.omega)}*t)"
        return (f"{r(self.amp)}*exp(-((x-{r(self.radius)}*cos({th}))**2"
                f"+(y-{r(self.radius)}*sin({th}))**2)/{r(self.width)}**2)")


_DTYPES = {torch.complex64: _lib.C64, torch.complex128: _lib.C128}


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dptr(values):
    arr = np.ascontiguousarray(values, dtype=np.float64)
    return arr, arr.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Plan:
    """One propagator configuration (``gpe_plan_create``).

    ``n``, ``x_array``, ``k_array``: grid (the reference's ``stage.N_grids``,
    ``x_array``, ``k_array``); ``dtype``: ``torch.complex64`` or ``complex128``;
    ``kind``: ``"imaginary"`` or ``"real"``; ``beta``, ``dt``, ``kinetic_coeff``:
    the step's coefficients (1.0 = the reference's ``exp(-i k^2 dt)``);
    ``static_expr`` / ``dynamic_expr``: potentials in the reference's expression
    grammar; ``k_cut``: momentum cutoff (real time); ``beam``: built-in stirring
    beam; ``nk_bins``: 0 = the reference's shell binning, else uniform bins.
    Options that keep results identical: ``path`` (``"default"``, ``"tma"``,
    ``"plane"`` or ``"auto"``: the sweep path, see ``tune.py``; ``tma`` and
    ``fuse_planes`` are the older switches for two of them) and
    ``generic_only`` (mixed-radix sweeps only).  Options that change results on
    purpose: ``local_fp64`` (complex64 local factor in FP64) and ``exact_local``
    (exact local sub-flows).
    """

    def __init__(self, n, x_array, k_array, *, dtype, kind, beta, dt, kinetic_coeff=1.0,
                 static_expr="0", dynamic_expr="0", k_cut=None, beam=None, nk_bins=0,
                 local_fp64=None, generic_only=False, fuse_planes=False, exact_local=False, tma=False,
                 path=None):
        if not torch.cuda.is_available():
            raise RuntimeError("gpe_simulator_b200 needs a CUDA device (sm_100a)")
        self.lib = _lib.load()
        self.n = int(n)
        self.dtype = dtype
        self.kind = kind
        if dtype not in _DTYPES:
            raise TypeError("psi must be complex64 or complex128")
        if kind not in ("imaginary", "real"):
            raise KeyError("kind must be 'imaginary' or 'real'")
        self.beta, self.dt, self.kinetic_coeff = float(beta), float(dt), float(kinetic_coeff)
        self.device = torch.cuda.current_device()
        x = np.asarray(torch.as_tensor(x_array).detach().cpu(), dtype=np.float64)
        k = np.asarray(torch.as_tensor(k_array).detach().cpu(), dtype=np.float64)
        if x.shape != (self.n,) or k.shape != (self.n,):
            raise AssertionError("x_array and k_array must have shape (N_grids,)")
        self.x, self.k = x, k
        keep = []
        d = _lib.Desc()
        d.n = self.n
        d.dtype = _DTYPES[dtype]
        d.kind = _lib.IMAGINARY if kind == "imaginary" else _lib.REAL
        d.beta, d.dt, d.kinetic_coeff = self.beta, self.dt, self.kinetic_coeff
        a, d.x_array = _dptr(x)
        keep.append(a)
        a, d.k_array = _dptr(k)
        keep.append(a)
        progs = dict(zip(("static_x", "static_y", "static_z", "static_g"), split_static(static_expr)))
        if kind == "real":
            progs["dynamic_g"] = compile_program(dynamic_expr, time_dependent=True)
        elif dynamic_expr not in ("0", None):
            raise ValueError("Imaginary time evolution does not accept a time dependent potential.")
        for name, prog in progs.items():
            if prog:
                a, ptr = _dptr(prog)
                keep.append(a)
                setattr(d, name, ptr)
                setattr(d, name + "_len", len(prog))
        if k_cut is not None:
            d.k_cut_enabled, d.k_cut = 1, float(k_cut)
        if beam is not None:
            d.beam_enabled = 1
            d.beam_amp, d.beam_width, d.beam_radius = beam.amp, beam.width, beam.radius
            d.beam_omega, d.beam_t_ramp = beam.omega, beam.t_ramp
        d.nk_bins = int(nk_bins)
        # complex64: FP32 phase evaluation by default (factor applied as v + v*(f - 1));
        # local_fp64=True evaluates the local factor in FP64 instead
        if local_fp64 is None:
            local_fp64 = False
        d.local_fp64 = 1 if local_fp64 else 0
        # sweep path: 0 fastest, 1 generic only, 3 y/z sweeps fused per x-plane (complex64 n = 128, 256),
        # 4 fastest with the y/x pencils staged by TMA (complex64 n = 128, 256; identical results).
        # ``path`` names it instead: "default", "tma", "plane", or "auto" (timed once per device,
        # size, dtype and kind, then cached; see tune.py)
        if path is not None:
            if path == "auto":
                from .tune import choose_path
                path = choose_path(self.n, x, k, dtype, kind)
            if path not in ("default", "tma", "plane"):
                raise ValueError("path must be 'default', 'tma', 'plane' or 'auto'")
            tma, fuse_planes = path == "tma", path == "plane"
        self.path = "plane" if fuse_planes else ("tma" if tma else "default")
        d.generic_only = 1 if generic_only else (3 if fuse_planes else (4 if tma else 0))
        # exact local sub-flows: an accuracy mode that departs from the reference on purpose
        d.exact_local = 1 if exact_local else 0
        self.local_fp64 = bool(local_fp64)
        handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(self.lib.gpe_plan_create(ctypes.byref(d), ctypes.byref(handle)))
        self._h = handle
        info = [ctypes.c_int() for _ in range(4)]
        self.lib.gpe_plan_info(self._h, *[ctypes.byref(v) for v in info])
        self.nbins = info[3].value
        self._static = None

    # ------------------------------------------------------------ lifetime
    def close(self):
        if getattr(self, "_h", None):
            torch.cuda.synchronize(self.device)
            self.lib.gpe_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------ checks
    def _check(self, t, name="psi"):
        if not isinstance(t, torch.Tensor):
            raise AssertionError(f"{name} must be a torch tensor")
        if not t.is_cuda or t.device.index != self.device:
            raise AssertionError(f"{name} must live on cuda:{self.device}")
        if t.dtype != self.dtype:
            raise AssertionError(f"{name} must be {self.dtype}")
        if not t.is_contiguous():
            raise AssertionError(f"{name} must be C-contiguous")
        if tuple(t.shape) != (self.n,) * 3:
            raise AssertionError(f"{name} must have shape (N_grids, N_grids, N_grids)")
        return ctypes.c_void_p(t.data_ptr())

    # ------------------------------------------------------------ potential
    def set_static_potential(self, v):
        """Static array potential (``stage.staticV``): float64 (imaginary) or
        complex128 ``U - i Gamma`` (real); ``None`` clears it."""
        if v is None:
            kind, ptr = _lib.V_NONE, None
        else:
            if not isinstance(v, torch.Tensor) or not v.is_cuda or tuple(v.shape) != (self.n,) * 3:
                raise AssertionError("staticV must be a CUDA tensor of shape (N_grids,)*3")
            if not v.is_contiguous():
                raise AssertionError("staticV must be C-contiguous")
            if v.dtype == torch.float64:
                kind = _lib.V_REAL64
            elif v.dtype == torch.complex128:
                if self.kind == "imaginary":
                    raise AssertionError("imaginary time requires a float64 staticV")
                kind = _lib.V_CPLX128
            else:
                raise AssertionError("staticV must be float64 or complex128")
            ptr = ctypes.c_void_p(v.data_ptr())
        _lib.check(self.lib.gpe_set_static_potential(self._h, ptr, kind, _stream()))
        self._static = v

    # ------------------------------------------------------------ propagation
    def step(self, psi, nsteps=1, step0=0):
        """``nsteps`` Strang steps in place; step ``i`` uses ``t = i*dt``."""
        p = self._check(psi)
        _lib.check(self.lib.gpe_step(self._h, p, int(nsteps), int(step0), _stream()))
        return psi

    def step_at(self, psi, t):
        """One Strang step whose half-steps use ``t + dt/2`` (closure semantics)."""
        p = self._check(psi)
        _lib.check(self.lib.gpe_step_at(self._h, p, float(t), _stream()))
        return psi

    def halfstep(self, psi, t):
        """The local half-step alone, at time ``t`` (kernel factories' contract)."""
        p = self._check(psi)
        _lib.check(self.lib.gpe_halfstep(self._h, p, float(t), _stream()))
        return psi

    def fft(self, src, out=None, inverse=False):
        """Unnormalised forward 3-D FFT, or inverse with 1/N^3 (``cp.fft.fftn/ifftn``)."""
        ps = self._check(src, "input")
        if out is None:
            out = torch.empty_like(src)
        po = self._check(out, "out")
        _lib.check(self.lib.gpe_fft3d(self._h, ps, po, 1 if inverse else 0, _stream()))
        return out

    def normalise(self, psi):
        p = self._check(psi)
        _lib.check(self.lib.gpe_normalise(self._h, p, _stream()))
        return psi

    # ------------------------------------------------------------ reductions (synchronous)
    def norm(self, psi):
        p = self._check(psi)
        out = ctypes.c_double()
        _lib.check(self.lib.gpe_norm(self._h, p, ctypes.byref(out), _stream()))
        return out.value

    def kinetic_energy(self, psi_k):
        p = self._check(psi_k, "psi_k")
        out = ctypes.c_double()
        _lib.check(self.lib.gpe_kinetic_energy(self._h, p, ctypes.byref(out), _stream()))
        return out.value

    def angular_momentum(self, psi):
        """Lz of ``psi`` (``gpe/helper.py:143-156``), FP64 sums."""
        p = self._check(psi)
        out = ctypes.c_double()
        _lib.check(self.lib.gpe_angular_momentum(self._h, p, ctypes.byref(out), _stream()))
        return out.value

    PROJECTIONS = ("TOF_xy", "TOF_yz", "TOF_slice_xy", "TOF_slice_yz", "density_xy", "density_slice_xy",
                   "phase_xy")

    def projections(self, psi, which=None):
        """Image outputs of ``gpe/save.py:59-90`` as ``{name: (n, n) array}``; ``which``
        is an iterable of names from :attr:`PROJECTIONS` (default: all)."""
        names = list(self.PROJECTIONS if which is None else which)
        bits = 0
        for name in names:
            bits |= 1 << self.PROJECTIONS.index(name)
        p = self._check(psi)
        chosen = [nm for nm in self.PROJECTIONS if bits >> self.PROJECTIONS.index(nm) & 1]
        out = np.empty((len(chosen), self.n, self.n))
        _lib.check(self.lib.gpe_projections(self._h, p, bits, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                            _stream()))
        return dict(zip(chosen, out))

    def shells(self, psi_k):
        """``(Nk, counts)`` per shell of a spectrum."""
        p = self._check(psi_k, "psi_k")
        nk = np.zeros(self.nbins)
        counts = np.zeros(self.nbins, np.int64)
        _lib.check(self.lib.gpe_nk_extraction(
            self._h, p, nk.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            counts.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)), _stream()))
        return nk, counts

    def diagnostics(self, psi, t=0.0, nk=False):
        """N, E_kin, E_pot, E_int, E, mu (+ Nk, counts) of ``psi`` at time ``t``."""
        p = self._check(psi)
        sc = np.zeros(6)
        nkv = np.zeros(self.nbins) if nk else None
        counts = np.zeros(self.nbins, np.int64) if nk else None
        _lib.check(self.lib.gpe_diagnostics(
            self._h, p, float(t), sc.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            nkv.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if nk else None,
            counts.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)) if nk else None, _stream()))
        out = dict(zip(("N", "E_kin", "E_pot", "E_int", "E", "mu"), map(float, sc)))
        if nk:
            out["Nk"], out["counts"] = nkv, counts
        return out

    def status(self):
        """Device status bits (1 = non-finite norm, 2 = timeout, 4 = a sweep refused its
        shared-memory layout); clears them."""
        flags = ctypes.c_int()
        _lib.check(self.lib.gpe_status(self._h, ctypes.byref(flags), _stream()))
        return flags.value


def oscillator_to_reference(V_scale=1.0):
    """Factors mapping oscillator units (kinetic ``exp(-i dt k^2/2)``) to the
    reference convention (``exp(-i k^2 dt)``): ``V_ref = 2 V``, ``beta = 2 g``,
    ``dt_ref = dt/2``, ``t_ref = t/2``."""
    return dict(potential=2.0 * V_scale, interaction=2.0, time=0.5)


def beam_in_reference_units(amp, width, radius, omega, ramp_time):
    """A beam given in oscillator units, expressed for a reference-unit plan."""
    return Beam(amp=2.0 * amp, width=width, radius=radius, omega=2.0 * omega, t_ramp=0.5 * ramp_time)


def reference_nbins(n):
    """``gpe/nk_extraction.py:21``."""
    return int(math.floor(math.sqrt(3) * (n // 2) + 0.5)) + 1


def launch_count(plan):
    """Kernel launches issued by ``plan`` since it was created."""
    out = ctypes.c_longlong()
    _lib.check(plan.lib.gpe_launch_count(plan._h, ctypes.byref(out)))
    return out.value


def profile(plan, enable):
    """Bracket each sweep launch of ``plan`` with CUDA events (or stop)."""
    _lib.check(plan.lib.gpe_profile(plan._h, 1 if enable else 0))


def profile_read(plan):
    """``{axis: (total_ms, launches)}`` for the sweeps recorded since :func:`profile`."""
    ms = np.zeros(3)
    cnt = np.zeros(3, np.int64)
    _lib.check(plan.lib.gpe_profile_read(plan._h, ms.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                         cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))))
    return {ax: (float(ms[i]), int(cnt[i])) for i, ax in enumerate(("z", "y", "x"))}
