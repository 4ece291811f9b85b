"""B200-native split-step Fourier propagator for the 3-D Gross-Pitaevskii equation.

A drop-in for the propagator path of PoyntingZhang/GPE_simulator
(``make_real_propagator`` / ``make_imag_propagator`` / ``stage`` /
``launch_stage``): Python host code over the C ABI of ``libgpe_ssf.so``
(``include/gpe_ssf.h``), hand-written CUDA for sm_100a, no cuFFT and no CPU
fallback.
"""

from .plan import Beam, Plan, beam_in_reference_units, reference_nbins  # noqa: F401

__all__ = ["Beam", "Plan", "beam_in_reference_units", "reference_nbins"]
