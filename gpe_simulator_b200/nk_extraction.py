"""Radial shell spectrum of ``|psi(k)|^2`` (``gpe/nk_extraction.py:16-45``).

The per-mode shell ids and weights are never materialised: a fused k-space
sweep accumulates per-block shell histograms in shared memory and a fixed-order
pass sums them.  Returned arrays are NumPy (they are small).
"""

import math

import numpy as np

from .helper import utility_plan


def shell_geometry(n, dk, nbins=None):
    """Bin count and width: reference (width dk, ``floor(sqrt3 (N//2) + 0.5) + 1``
    bins) or ``nbins`` uniform bins reaching the cube corner."""
    if not nbins:
        return int(math.floor(math.sqrt(3) * (n // 2) + 0.5)) + 1, dk
    return int(nbins), math.sqrt(3) * (n // 2) * dk / (int(nbins) - 1)


def assemble(Nk, counts, n, dk, nbins=None):
    """The reference's output dictionary from per-shell ``Nk`` and ``counts``."""
    nb, width = shell_geometry(n, dk, nbins)
    nk = Nk / (np.maximum(counts, 1) * dk ** 3)
    k = np.arange(nb, dtype=np.float64) * width
    edges = (np.arange(nb + 1, dtype=np.float64) - 0.5) * width
    edges[0] = 0
    complete = edges[1:] <= n * dk / 2
    return dict(k=k, nk=nk, Nk=Nk, counts=counts, edges=edges, complete_shells=complete)


def nk_extraction(psi_k, x_array, k_array, slab_size=16, nbins=None):
    """Shell averages from raw ``fftn(psi)``; ``Nk`` sums to the norm.

    ``slab_size`` is accepted for signature compatibility; the fused sweep has
    no slabs.  ``nbins`` selects the uniform-bin extension.
    """
    n = psi_k.shape[0]
    ks = k_array.detach().cpu().numpy()
    dk = abs(float(ks[1] - ks[0]))
    plan = utility_plan(psi_k, x_array, k_array, nbins=nbins or 0)
    Nk, counts = plan.shells(psi_k)
    return assemble(Nk, counts, n, dk, nbins)
