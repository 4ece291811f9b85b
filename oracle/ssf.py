"""FP64 NumPy/scipy.fft restatement of the reference split-step propagator.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``): the checker for the CUDA
path and the CPU baseline of ``bench.py``.  It is never imported by the
product package.

Conventions follow the reference exactly (reference units):

* Hamiltonian ``i dpsi/dt = [-c_kin lap + V + beta |psi|^2] psi`` with
  ``c_kin = 1`` in the reference (kinetic factor ``exp(-i k^2 dt)``,
  ``gpe/kernels.py:3-21``).  ``c_kin = 0.5`` is the oscillator-unit convention;
  it is an extension.
* ``x = linspace(-L/2, L/2, N, endpoint=False)``, ``k = 2 pi fftfreq(N, L/N)``
  (``gpe/grids.py:3-6``); arrays are ``[x][y][z]`` C-order.
* one step = local half-step -> fftn -> kinetic -> ifftn -> local half-step, and
  for imaginary time a renormalisation (``gpe/make_propagator.py:12-54``,
  ``57-103``, ``109-151``).  Dynamic potentials are evaluated at
  ``t_mid = t + dt/2`` for both halves (``gpe/make_propagator.py:94-101``) with
  ``t = i*dt`` (``gpe/launch.py:10``).
"""

from dataclasses import dataclass, field
import math
import os

import numpy as np
import scipy.fft as sfft

from . import expr

WORKERS = int(os.environ.get("GPE_ORACLE_WORKERS", os.cpu_count() or 1))


def fftn(a):
    return sfft.fftn(a, workers=WORKERS)


def ifftn(a):
    return sfft.ifftn(a, workers=WORKERS)


# --------------------------------------------------------------------------- grids
def get_grids(n, simulation_range):
    """``gpe/grids.py:3-6``."""
    x = np.linspace(-simulation_range / 2, simulation_range / 2, n, endpoint=False)
    k = 2 * np.pi * np.fft.fftfreq(n, simulation_range / n)
    return x, k


def get_beta(n_atoms, a):
    """``gpe/helper.py:109-113`` (a in Bohr radii, l = 1 micrometre)."""
    return 8 * np.pi * n_atoms * (a * 5.29177210544e-11) / 1e-6


# --------------------------------------------------------------------------- norm
def get_N(psi, x):
    """``gpe/helper.py:81-88``: ``dx^3 sum |psi|^2`` in FP64."""
    dx = x[1] - x[0]
    return float(np.sum(np.abs(psi.astype(np.complex128)) ** 2)) * dx ** 3


def normalise(psi, x):
    """``gpe/helper.py:91-93``: ``psi /= sqrt(N)`` (in place)."""
    psi /= np.sqrt(get_N(psi, x))
    return psi


def gaussian(x, sigma):
    """``gpe/initial_states.py:4-14``: normalised separable Gaussian."""
    g = np.exp(-x ** 2 / (2 * sigma ** 2)).astype(np.complex128)
    psi = g[:, None, None] * g[None, :, None] * g[None, None, :]
    return normalise(psi, x)


def noisy_gaussian(x, sigma=1.0, eps=0.01, seed=0):
    """Seeded Gaussian x (1 + eps xi), xi complex standard normal, normalised.

    ``xi = (a + i b)/sqrt(2)`` with ``a`` then ``b`` drawn from
    ``default_rng(seed).standard_normal((N,N,N))`` in C order.
    """
    n = len(x)
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n, n))
    b = rng.standard_normal((n, n, n))
    g = np.exp(-x ** 2 / (2 * sigma ** 2))
    psi = (g[:, None, None] * g[None, :, None] * g[None, None, :]) * (1 + eps * (a + 1j * b) / np.sqrt(2))
    return normalise(psi.astype(np.complex128), x)


# --------------------------------------------------------------------------- model
@dataclass
class Beam:
    """Rotating Gaussian stirring beam (reference units).

    ``V = amp * exp(-((x - r0 cos th)^2 + (y - r0 sin th)^2) / w^2)`` with the
    angular rate ramped linearly from 0 to ``omega`` over ``t_ramp``:
    ``th(t) = omega * (m^2 / (2 t_ramp) + t - m)``, ``m = min(t, t_ramp)``.
    """
    amp: float
    width: float
    radius: float
    omega: float
    t_ramp: float = 0.0

    def theta(self, t):
        if self.t_ramp > 0:
            m = min(t, self.t_ramp)
            return self.omega * (m * m / (2 * self.t_ramp) + t - m)
        return self.omega * t

    def value(self, X, Y, t):
        th = self.theta(t)
        cx, cy = self.radius * math.cos(th), self.radius * math.sin(th)
        return self.amp * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / self.width ** 2)

    def expression(self):
        """The same beam in the reference's potential grammar."""
        m = f"((t+{self.t_ramp!r}-abs(t-{self.t_ramp!r}))/2)"
        if self.t_ramp > 0:
            th = f"({self.omega!r}*({m}**2/(2*{self.t_ramp!r})+t-{m}))"
        else:
            th = f"({self.omega!r}*t)"
        return (f"{self.amp!r}*exp(-((x-{self.radius!r}*cos({th}))**2"
                f"+(y-{self.radius!r}*sin({th}))**2)/{self.width!r}**2)")


@dataclass
class Model:
    """Everything one propagator step reads from a reference ``stage``.

    ``gpe/stage.py:12-51`` + ``gpe/make_kernel.py`` (expressions) +
    ``gpe/kernels.py`` (kinetic, optional cutoff).
    """
    n: int
    simulation_range: float
    kind: str                     # "imaginary" | "real"
    beta: float
    dt: float
    ckin: float = 1.0
    static_expr: str = "0"
    dynamic_expr: str = "0"
    static_v: np.ndarray = None   # real (imag time) or complex U - i Gamma (real time)
    k_cut: float = None
    beam: Beam = None
    exact_local: bool = False     # exact local sub-flows (not the reference's; parity off)
    x: np.ndarray = field(init=False)
    k: np.ndarray = field(init=False)

    def __post_init__(self):
        self.x, self.k = get_grids(self.n, self.simulation_range)

    @property
    def dx(self):
        return self.x[1] - self.x[0]

    def axes(self):
        return self.x[:, None, None], self.x[None, :, None], self.x[None, None, :]

    def k2(self):
        k = self.k
        return k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2

    def potential(self, t):
        """Real potential ``Re V_static + V_expr + V_dyn(t) + beam(t)``."""
        X, Y, Z = self.axes()
        v = np.zeros((self.n,) * 3)
        if self.static_v is not None:
            v = v + np.real(self.static_v)
        v = v + expr.evaluate(self.static_expr, X, Y, Z)
        if self.kind == "real":
            v = v + expr.evaluate(self.dynamic_expr, X, Y, Z, t, time_dependent=True)
            if self.beam is not None:
                v = v + self.beam.value(X, Y, t)
        return np.broadcast_to(v, (self.n,) * 3)

    def loss(self):
        """``Im V_static`` (``-Gamma``) for real time, else 0."""
        if self.kind == "real" and self.static_v is not None and np.iscomplexobj(self.static_v):
            return np.imag(self.static_v)
        return 0.0


# --------------------------------------------------------------------------- kernels
def halfstep(psi, model, t_mid=0.0):
    """Local half-step, in place.

    real: ``gpe/make_kernel.py:14-45`` / ``54-83``:
        ``psi *= exp(ImV dt/2 - i (ReV + beta|psi|^2 + V_expr) dt/2)``
    imaginary: ``gpe/make_kernel.py:93-119``:
        ``psi *= exp(-(V + beta|psi|^2 + V_expr) dt/2)``
    """
    v = model.potential(t_mid)
    h = model.dt / 2
    rdt = np.float64 if psi.dtype == np.complex128 else np.float32
    abs2 = psi.real.astype(np.float64) ** 2 + psi.imag.astype(np.float64) ** 2
    if model.exact_local:
        # exact flows of the local subproblem with V fixed over h (the reference's
        # notes, "GPE simulator/HANDOFF.md" accepted approximations): imaginary time
        # psi e^{-Vh}/sqrt(1 + 2 beta|psi|^2 s); real time with Gamma = -Im V,
        # phase Vh + beta|psi|^2 tau and amplitude e^{-Gamma h}
        with np.errstate(divide="ignore", invalid="ignore"):
            if model.kind == "imaginary":
                s = np.where(v == 0, h, -np.expm1(-2 * v * h) / (2 * v))
                psi *= (np.exp(-v * h) / np.sqrt(1 + 2 * model.beta * abs2 * s)).astype(rdt)
            else:
                g = -np.broadcast_to(model.loss(), v.shape)
                tau = np.where(g == 0, h, -np.expm1(-2 * g * h) / (2 * g))
                psi *= np.exp(-g * h - 1j * (v * h + model.beta * abs2 * tau)).astype(psi.dtype)
        return psi
    phase = (v + model.beta * abs2) * h
    if model.kind == "imaginary":
        psi *= np.exp(-phase).astype(rdt)
    else:
        psi *= np.exp(model.loss() * h - 1j * phase).astype(psi.dtype)
    return psi


def kinetic(psi_k, model):
    """Kinetic full step on ``fftn(psi)``, in place.

    real ``gpe/kernels.py:3-21`` (``exp(-i k^2 dt)``), with cutoff
    ``gpe/kernels.py:24-45`` (modes with ``k^2 > k_cut^2`` set to 0), imaginary
    ``gpe/kernels.py:48-66`` (``exp(-k^2 dt)``); ``k^2`` scaled by ``ckin``.
    """
    k2 = model.k2()
    phase = model.ckin * k2 * model.dt
    if model.kind == "imaginary":
        factor = np.exp(-phase)
    else:
        factor = np.exp(-1j * phase)
        if model.k_cut is not None:
            factor = np.where(k2 > model.k_cut ** 2, 0.0, factor)
    psi_k *= factor.astype(psi_k.dtype)
    return psi_k


def step(psi, model, t=0.0):
    """One Strang step (``gpe/make_propagator.py``); returns the new array."""
    t_mid = float(t) + model.dt / 2
    halfstep(psi, model, t_mid)
    psi_k = fftn(psi)
    kinetic(psi_k, model)
    psi = ifftn(psi_k)
    halfstep(psi, model, t_mid)
    if model.kind == "imaginary":
        normalise(psi, model.x)
    return psi


def run(psi, model, steps, step0=0):
    """``gpe/launch.py:8-13`` without outputs: step ``i`` uses ``t = i*dt``."""
    psi = np.array(psi, copy=True)
    for i in range(step0, step0 + steps):
        psi = step(psi, model, i * model.dt)
    return psi


# --------------------------------------------------------------------------- diagnostics
def get_E(psi_k, x, k):
    """``gpe/helper.py:135-140``: ``E_kin = dx^3/M sum k^2 |F|^2``."""
    dx = x[1] - x[0]
    k2 = k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2
    return float(np.sum(np.abs(psi_k.astype(np.complex128)) ** 2 * k2)) * dx ** 3 / psi_k.size


def get_L(psi, x, k, slab_size=16):
    """``gpe/helper.py:143-156``: ``Lz = dx^3 sum [x Re(psi* P_y psi) - y Re(psi* P_x psi)]``
    with spectral momenta ``P = ifftn(k fftn(.))`` over the (x, y) axes of z slabs."""
    dx = x[1] - x[0]
    L = 0.0
    for start in range(0, psi.shape[2], slab_size):
        slab = psi[:, :, start:start + slab_size].astype(np.complex128)
        sk = np.fft.fftn(slab, axes=(0, 1))
        my = np.fft.ifftn(sk * k[None, :, None], axes=(0, 1))
        L += float(np.sum(x[:, None, None] * (slab.real * my.real + slab.imag * my.imag)))
        mx = np.fft.ifftn(sk * k[:, None, None], axes=(0, 1))
        L -= float(np.sum(x[None, :, None] * (slab.real * mx.real + slab.imag * mx.imag)))
    return L * dx ** 3


PROJECTIONS = ("TOF_xy", "TOF_yz", "TOF_slice_xy", "TOF_slice_yz", "density_xy", "density_slice_xy",
               "phase_xy")


def projections(psi, x, k):
    """The image outputs of ``gpe/save.py:59-90`` (values only): momentum-space
    (time-of-flight) column sums over z and x and the kz = 0 / kx = 0 slices of
    ``|fftn(psi)|^2``, fftshifted and scaled by ``dx^3/(M dk^3)`` (columns also by
    ``dk``); the real-space column density over z (times dx), the z = N/2 slice
    of ``|psi|^2`` and its phase (NaN where the slice density is below 1e-12 of
    its maximum)."""
    psi = psi.astype(np.complex128)
    n = psi.shape[0]
    dx = float(x[1] - x[0])
    dk = abs(float(k[1] - k[0]))
    F = np.fft.fftn(psi)
    w = np.abs(F) ** 2
    scale = dx ** 3 / (psi.size * dk ** 3)
    sh = np.fft.fftshift
    out = dict(TOF_xy=sh(w.sum(axis=2)) * (scale * dk), TOF_yz=sh(w.sum(axis=0)) * (scale * dk),
               TOF_slice_xy=sh(w[:, :, 0]) * scale, TOF_slice_yz=sh(w[0, :, :]) * scale)
    out["density_xy"] = (np.abs(psi) ** 2).sum(axis=2) * dx
    plane = psi[:, :, n // 2]
    dens = np.abs(plane) ** 2
    out["density_slice_xy"] = dens
    out["phase_xy"] = np.where(dens > dens.max() * 1e-12, np.angle(plane), np.nan)
    return out


def reference_nbins(n):
    """``gpe/nk_extraction.py:21``."""
    return int(math.floor(math.sqrt(3) * (n // 2) + 0.5)) + 1


def nk_extraction(psi_k, x, k, nbins=None):
    """``gpe/nk_extraction.py:16-45``; ``nbins`` selects the uniform-width extension.

    Reference binning: shell width ``dk = 2 pi / L``, ``shell = floor(|k|/dk + 0.5)``.
    Extension (``nbins`` given): width ``kmax / (nbins - 1)`` with
    ``kmax = sqrt(3) (N//2) dk`` so the cube corner falls in the last bin.
    """
    n = psi_k.shape[0]
    dx = float(x[1] - x[0])
    dk = abs(float(k[1] - k[0]))
    if nbins is None:
        nbins = reference_nbins(n)
        width = dk
    else:
        width = math.sqrt(3) * (n // 2) * dk / (nbins - 1)
    kk = k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2
    shell = np.floor(np.sqrt(kk) / width + 0.5).astype(np.int64)
    shell = np.minimum(shell, nbins - 1)
    w = np.abs(psi_k.astype(np.complex128)) ** 2
    counts = np.bincount(shell.ravel(), minlength=nbins)
    occupation = np.bincount(shell.ravel(), weights=w.ravel(), minlength=nbins)
    Nk = occupation * (dx ** 3 / psi_k.size)
    nk = Nk / (np.maximum(counts, 1) * dk ** 3)
    kc = np.arange(nbins, dtype=np.float64) * width
    edges = (np.arange(nbins + 1, dtype=np.float64) - 0.5) * width
    edges[0] = 0
    complete = edges[1:] <= n * dk / 2
    return dict(k=kc, nk=nk, Nk=Nk, counts=counts, edges=edges, complete_shells=complete)


def energies(psi, model, t=0.0):
    """N, E_kin and the new total-energy diagnostics (parity unpinned).

    ``E_kin = ckin dx^3/M sum k^2 |F|^2`` (reference ``get_E`` for ckin = 1),
    ``E_pot = dx^3 sum V |psi|^2``, ``E_int = beta/2 dx^3 sum |psi|^4``,
    ``E = E_kin + E_pot + E_int``, ``mu = (E_kin + E_pot + 2 E_int) / N``.
    """
    psi = psi.astype(np.complex128)
    dx3 = model.dx ** 3
    rho = np.abs(psi) ** 2
    N = float(np.sum(rho)) * dx3
    e_kin = model.ckin * get_E(fftn(psi), model.x, model.k)
    e_pot = float(np.sum(model.potential(t) * rho)) * dx3
    e_int = 0.5 * model.beta * float(np.sum(rho * rho)) * dx3
    E = e_kin + e_pot + e_int
    return dict(N=N, E_kin=e_kin, E_pot=e_pot, E_int=e_int, E=E,
                mu=(e_kin + e_pot + 2 * e_int) / N)


def rel_l2(a, b):
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))
