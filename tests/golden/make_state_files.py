"""Generate ``tests/golden/state_ref/``: a snapshot written by the reference's own
``save_wavefunction`` (``gpe/state_io.py:14-28``).

Runs ONLY where ``GPE_REFERENCE`` names the reference's source tree; the
reference is imported on the host with its NumPy-backed CuPy
(``oracle/ref_shim.py``).  The state is the seeded 8^3 complex128 cube of
``tests/test_state_io.py::make_stage`` saved at step 4, so the files pin the
.npy bytes, the metadata text and the axes that the reference writes.

Usage: ``GPE_REFERENCE=<tree> python tests/golden/make_state_files.py``.
"""

import sys
from pathlib import Path
from types import SimpleNamespace

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import ref_shim  # noqa: E402

OUT = Path(__file__).resolve().parent / "state_ref"


def seeded_state(n=8, L=6.0):
    """The cube and axes of ``make_stage`` (torch's seeded generator, complex128)."""
    import torch
    x = np.linspace(-L / 2, L / 2 - L / n, n)
    k = 2 * np.pi * np.fft.fftfreq(n, L / n)
    g = torch.Generator().manual_seed(0)
    psi = torch.randn((n, n, n), dtype=torch.complex128, generator=g).numpy()
    return psi, x, k


def main():
    if not ref_shim.available():
        raise SystemExit(ref_shim.UNSET if ref_shim.REFERENCE is None else "the reference sources are not present")
    ref = ref_shim.install()
    psi, x, k = seeded_state()
    stage = SimpleNamespace(psi=psi, x_array=x, k_array=k, N_grids=8, dt=0.01, type="real", N_atoms=1000,
                            simulation_range=6.0, config={"name": "test"})
    OUT.mkdir(exist_ok=True)
    ref.state_io.save_wavefunction(OUT / "psi_00000004.npy", stage, 4)
    for f in sorted(OUT.iterdir()):
        print("wrote", f.relative_to(ROOT), f.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
