"""Grids, norm, normalisation, energies and scheduling helpers.

Drop-in counterparts of ``gpe/grids.py``, ``gpe/helper.py`` and
``gpe/initial_states.py``, on torch CUDA tensors.  Reductions and FFTs run in
``libgpe_ssf.so`` through a cached utility plan per (grid, dtype, device).
"""

from collections import OrderedDict
import math

import numpy as np
import torch

from .plan import Plan

# utility plans by (grid, dtype, device, shell binning), least recently used first;
# the oldest is dropped once more than _UTIL_MAX are held (a plan frees its tables when
# no caller holds it any more)
_UTIL = OrderedDict()
_UTIL_MAX = 16


def get_grids(N_grids, simulation_range, device="cuda"):
    """``gpe/grids.py:3-6``: x on [-L/2, L/2) and ``k = 2 pi fftfreq(N, L/N)`` (float64)."""
    x = np.linspace(-simulation_range / 2, simulation_range / 2, N_grids, endpoint=False)
    k = 2 * np.pi * np.fft.fftfreq(N_grids, simulation_range / N_grids)
    return torch.from_numpy(x).to(device), torch.from_numpy(k).to(device)


def utility_plan(psi, x_array, k_array=None, nbins=0):
    """Plan without physics, for FFTs and reductions on ``psi``'s grid (``nbins``:
    0 = the reference's shell binning, else that many uniform bins).  Plans are
    cached, so repeated diagnostics on one grid create no new device tables."""
    n = psi.shape[0]
    xs = x_array.detach().cpu().numpy() if isinstance(x_array, torch.Tensor) else np.asarray(x_array)
    if k_array is None:
        L = (xs[1] - xs[0]) * n
        ks = 2 * np.pi * np.fft.fftfreq(n, L / n)
    else:
        ks = k_array.detach().cpu().numpy() if isinstance(k_array, torch.Tensor) else np.asarray(k_array)
    key = (n, psi.dtype, psi.device.index, float(xs[0]), float(xs[1]), float(ks[1]), int(nbins or 0))
    plan = _UTIL.get(key)
    if plan is None:
        with torch.cuda.device(psi.device):
            plan = Plan(n, xs, ks, dtype=psi.dtype, kind="imaginary", beta=0.0, dt=0.0, nk_bins=int(nbins or 0))
        _UTIL[key] = plan
        while len(_UTIL) > _UTIL_MAX:
            _UTIL.popitem(last=False)
    else:
        _UTIL.move_to_end(key)
    return plan


def fftn(psi, x_array=None):
    """Unnormalised forward 3-D FFT of a cube (``cp.fft.fftn``)."""
    x = x_array if x_array is not None else torch.linspace(-1, 1, psi.shape[0] + 1)[:-1]
    return utility_plan(psi, x).fft(psi)


def ifftn(psi_k, x_array=None):
    """Inverse 3-D FFT with 1/N^3 (``cp.fft.ifftn``)."""
    x = x_array if x_array is not None else torch.linspace(-1, 1, psi_k.shape[0] + 1)[:-1]
    return utility_plan(psi_k, x).fft(psi_k, inverse=True)


def get_N(psi, x_array):
    """``gpe/helper.py:81-88``: ``dx^3 sum |psi|^2`` (FP64, compensated)."""
    return utility_plan(psi, x_array).norm(psi)


def normalise(psi, x_array):
    """``gpe/helper.py:91-93``: ``psi /= sqrt(N)`` in place."""
    utility_plan(psi, x_array).normalise(psi)
    return psi


def get_E(psi_k, x_array, k_array):
    """``gpe/helper.py:135-140``: ``dx^3/M sum k^2 |F|^2`` of ``F = fftn(psi)``."""
    return utility_plan(psi_k, x_array, k_array).kinetic_energy(psi_k)


def get_L(psi, x_array, k_array, slab_size=16):
    """``gpe/helper.py:143-156``: ``Lz = Re integral psi* (x p_y - y p_x) psi dV`` with
    spectral momenta (``slab_size`` is accepted for the reference's signature; the
    sums here need no slabs)."""
    return utility_plan(psi, x_array, k_array).angular_momentum(psi)


def get_beta(N_atoms, a):
    """``gpe/helper.py:109-113`` (a in Bohr radii, l = 1 micrometre)."""
    return 8 * math.pi * N_atoms * (a * 5.29177210544e-11) / 1e-6


def is_due(i, interval):
    """``gpe/helper.py:131-132``."""
    return i > 0 and interval is not None and interval > 0 and i % interval == 0


def gaussian(x_array, sigma, dtype=torch.complex128):
    """``gpe/initial_states.py:4-14``: normalised separable Gaussian."""
    g = torch.exp(-x_array.to(torch.float64) ** 2 / (2 * sigma ** 2)).to(torch.complex128)
    psi = (g[:, None, None] * g[None, :, None] * g[None, None, :]).to(dtype).contiguous()
    return normalise(psi, x_array)
