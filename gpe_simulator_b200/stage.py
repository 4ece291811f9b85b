"""State container of one simulation stage (``gpe/stage.py``), torch-backed.

Same constructor, attributes and ``prepare``/``release`` contract as the
reference; ``x_array``/``k_array`` are float64 CUDA tensors from
:func:`gpe_simulator_b200.helper.get_grids`.  Extensions (keyword-only):
``precision`` ("complex128" as in the reference, or "complex64"),
``kinetic_coeff`` (1.0 = reference convention), ``beam`` (built-in stirring
beam) and ``nk_bins`` (uniform n(k) shells).
"""

import numpy as np
import torch

from .helper import gaussian, get_beta
from .make_propagator import make_imag_propagator, make_real_propagator

_PRECISION = {"complex128": torch.complex128, "complex64": torch.complex64}


def box_potential(x_grid, box_radius, box_length, wall_thickness, trap_depth):
    """Gaussian tube and end-cap walls (``gpe/potentials.py:3-11``), float64."""
    X, Y, Z = x_grid[:, None, None], x_grid[None, :, None], x_grid[None, None, :]
    tube = torch.exp(-(torch.sqrt(X ** 2 + Y ** 2) - box_radius) ** 2 / (2 * wall_thickness ** 2))
    sheet = torch.exp(-(torch.abs(Z) - box_length / 2) ** 2 / (2 * wall_thickness ** 2))
    return (torch.maximum(tube, sheet) * trap_depth).contiguous()


def absorption_potential(activation_distance, amplitude, x_grid, simulation_range):
    """Linear absorber ramps at the faces (``gpe/potentials.py:13-28``), float64."""
    X, Y, Z = x_grid[:, None, None], x_grid[None, :, None], x_grid[None, None, :]
    r = lambda v: torch.clamp(v, min=0)  # noqa: E731
    half = simulation_range / 2
    xy = r(activation_distance - (X + half)) + r(activation_distance - (half - X)) + \
        r(activation_distance - (Y + half)) + r(activation_distance - (half - Y))
    z = r(activation_distance - (Z + half)) + r(activation_distance - (half - Z))
    return ((xy + z) * amplitude).contiguous()


def total_static_potential(real_grid, imag_grid):
    """``U - i Gamma`` as complex128 (``gpe/potentials.py:31-37``)."""
    return torch.complex(real_grid.expand_as(imag_grid).contiguous(), -imag_grid).contiguous()


class stage:  # noqa: N801 -- the reference's class name
    def __init__(self, simulation_range, x_array, k_array, N_grids, type, steps, dt,
                 initial_state, box_params, absorber_params, noise_params, cloud_params,
                 monitor_params, save_params, potential_params, k_cut_params, *,
                 precision="complex128", kinetic_coeff=1.0, beam=None, nk_bins=0):
        if not isinstance(x_array, torch.Tensor):
            raise TypeError("x_array should be a torch tensor")
        if not isinstance(k_array, torch.Tensor):
            raise TypeError("k_array should be a torch tensor")
        if x_array.dtype != torch.float64:
            raise TypeError("x_array should be a real array")
        if k_array.dtype != torch.float64:
            raise TypeError("k_array should be a real array")
        if not isinstance(type, str):
            raise TypeError("type of the stage should be a string")
        if type not in {"imaginary", "real"}:
            raise KeyError("type of the stage should either be 'real' or 'imaginary")
        if precision not in _PRECISION:
            raise KeyError("precision should be 'complex128' or 'complex64'")
        self.absorber_params = absorber_params
        self.noise_params = noise_params
        self.simulation_range = simulation_range
        self.x_array = x_array
        self.k_array = k_array
        self.N_grids = N_grids
        self.type = type
        self.steps = steps
        self.dt = dt
        self.initial_state = initial_state
        self.box_params = box_params
        self.a = cloud_params["a"]
        self.N_atoms = cloud_params["N_atom"]
        self.save_params = save_params
        self.monitor_params = monitor_params
        self.potential_params = potential_params
        self.beta = get_beta(self.N_atoms, self.a)
        self.k_cut_params = k_cut_params
        self.precision = precision
        self.kinetic_coeff = kinetic_coeff
        self.beam = beam
        self.nk_bins = nk_bins
        self.psi = None
        self.staticV = None
        self.propagator = None
        self.name = ""
        self.config = {}

    def prepare(self, previous_psi=None):
        """Allocate psi and the static potential when the stage is about to run."""
        self.psi = self._get_initial_state(previous_psi)
        if self.type == "imaginary":
            self.staticV = self._get_box()
        else:
            self.staticV = total_static_potential(self._get_box(), self._get_absorber())
        if self.noise_params.get("activate"):
            self._add_white_noise()
        if self.type == "real":
            self.propagator = make_real_propagator(self)
        else:
            self.propagator = make_imag_propagator(self)

    def release(self):
        self.psi = None
        self.staticV = None
        self.propagator = None

    def _shape(self):
        return (self.N_grids,) * 3

    def _get_initial_state(self, previous_psi):
        kind = self.initial_state["type"]
        dtype = _PRECISION[self.precision]
        if kind == "continue":
            if previous_psi is None:
                raise ValueError("A continue stage needs the preceding stage's wavefunction.")
            return previous_psi.to(dtype).contiguous()
        if kind == "load":
            from .state_io import load_wavefunction
            return load_wavefunction(self.initial_state["path"], self, dtype)
        if kind == "gaussian":
            return gaussian(self.x_array, self.initial_state["sigma"], dtype=dtype)
        raise ValueError(f"Unknown initial state: {kind}")

    def _get_box(self):
        if not self.box_params["activate"]:
            return torch.zeros(self._shape(), dtype=torch.float64, device=self.x_array.device)
        b = self.box_params
        return box_potential(self.x_array, b["R"], b["L"], b["wall_thickness"], b["trap_depth"])

    def _get_absorber(self):
        if self.absorber_params["activate"]:
            a = self.absorber_params
            return absorption_potential(a["activation_distance"], a["strength"], self.x_array,
                                        self.simulation_range)
        return torch.zeros(self._shape(), dtype=torch.float64, device=self.x_array.device)

    def _add_white_noise(self):
        """Disorder ``N(0, (fraction * trap_depth)^2)`` added to ``Re staticV``
        (``gpe/potentials.py:39-61``); seeded torch generator, so the draws differ
        from CuPy's."""
        g = torch.Generator(device=self.x_array.device)
        g.manual_seed(int(self.noise_params.get("seed", 42)))
        sigma = float(self.noise_params["fraction"] * self.box_params["trap_depth"])
        noise = torch.randn(self._shape(), generator=g, dtype=torch.float64, device=self.x_array.device)
        if self.staticV.is_complex():
            self.staticV.real.add_(noise * sigma)
        else:
            self.staticV.add_(noise * sigma)
