"""Wavefunction snapshots in the reference's format (``gpe/state_io.py:14-58``).

A snapshot is a complex128 ``.npy`` cube written slab by slab (16 x-planes per
device-to-host transfer) through a memory map, ``grid.npz`` beside it with the
axes, and a ``.json`` file with the step, time, evolution type, reference atom
number, box size, grid size and the stage configuration.  A complex64 state is
widened to complex128 on the device, one slab at a time, before the transfer;
loading narrows on the device after the host-to-device copy of each slab.  Files
written here load in the reference and the other way round.
"""

import json
from pathlib import Path

import numpy as np
import torch

# x-planes per transfer (256 MiB for a 1024^3 complex128 grid)
SLAB_SIZE = 16


def _host(a):
    return a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)


def save_wavefunction(path, stage, step):
    """``gpe/state_io.py:14-29``: write ``stage.psi`` (any precision) as complex128."""
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    psi = stage.psi
    n = int(stage.N_grids)
    saved = np.lib.format.open_memmap(path, mode="w+", dtype=np.complex128, shape=(n, n, n))
    for start in range(0, n, SLAB_SIZE):
        saved[start:start + SLAB_SIZE] = psi[start:start + SLAB_SIZE].to(torch.complex128).cpu().numpy()
    saved.flush()
    del saved
    np.savez(path.parent / "grid.npz", x_array=_host(stage.x_array), k_array=_host(stage.k_array))
    metadata = dict(step=step, time=step * stage.dt, evolution=stage.type, N_atom=stage.N_atoms,
                    simulation_range=stage.simulation_range, N_grids=n, stage=getattr(stage, "config", {}))
    path.with_suffix(".json").write_text(json.dumps(metadata, indent=2) + "\n")


def load_wavefunction(path, stage, dtype=torch.complex128):
    """``gpe/state_io.py:32-58``: a saved complex128 cube matching the stage's grid,
    box and atom number, uploaded slab by slab and narrowed on the device to
    ``dtype``; its norm and clock are not changed."""
    path = Path(path)
    saved = np.load(path, mmap_mode="r", allow_pickle=False)
    n = int(stage.N_grids)
    if saved.shape != (n,) * 3 or saved.dtype != np.complex128:
        raise ValueError("The loaded state must be a complex128 cube matching N_grids.")
    metadata_path = path.with_suffix(".json")
    if metadata_path.exists():
        metadata = json.loads(metadata_path.read_text())
        if metadata["simulation_range"] != stage.simulation_range:
            raise ValueError("The loaded state has a different simulation range.")
        if metadata["N_atom"] != stage.N_atoms:
            raise ValueError("The loaded state uses a different reference N_atom.")
    # older exports keep the axes beside each snapshot rather than per directory
    grid_path = path.with_name(path.stem + "_grid.npz")
    if not grid_path.exists():
        grid_path = path.parent / "grid.npz"
    if grid_path.exists():
        with np.load(grid_path, allow_pickle=False) as grid:
            for name in ("x_array", "k_array"):
                expected = _host(getattr(stage, name))
                if grid[name].shape != expected.shape or not np.allclose(grid[name], expected):
                    raise ValueError("The loaded state's grid does not match this simulation.")
    device = stage.x_array.device if isinstance(stage.x_array, torch.Tensor) else torch.device("cpu")
    psi = torch.empty((n, n, n), dtype=dtype, device=device)
    for start in range(0, n, SLAB_SIZE):
        slab = torch.from_numpy(np.array(saved[start:start + SLAB_SIZE]))   # writable host copy of the slab
        psi[start:start + SLAB_SIZE] = slab.to(device).to(dtype)
    del saved
    return psi
