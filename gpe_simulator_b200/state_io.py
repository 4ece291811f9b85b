"""Wavefunction snapshots in the reference's file format.

The format is what must match (files written here load in the reference and
the other way round, ``gpe/state_io.py:14-58``): a complex128 ``.npy`` cube
``[x][y][z]``, ``grid.npz`` beside it with ``x_array`` and ``k_array``, and a
``.json`` file with ``step, time, evolution, N_atom, simulation_range, N_grids,
stage``.  A load accepts a file only when the cube matches ``N_grids``, the
metadata (when present) matches the stage's box and reference atom number, and
the axes (``<name>_grid.npz``, else ``grid.npz``, when present) match the
stage's grid.

The transfer is built for large cubes on a GPU.  The ``.npy`` header is written
and parsed here, and the data streams through the file in slabs of whole
x-planes of about 64 MiB: on the device a slab is widened to (or, on load,
narrowed from) complex128, and two pinned host buffers alternate, so that the
device-to-host copy of one slab runs while the other is written to the file
(on load: the file read of the next slab runs while the previous one is copied
to the device).  Host (CPU) tensors take the same slab loop without the copies.
"""

import json
from pathlib import Path

import numpy as np
import torch

_SLAB_BYTES = 64 << 20
_NPY_C128 = {"descr": np.dtype(np.complex128).str, "fortran_order": False}


def _host(a):
    return a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)


def _planes_per_slab(n):
    return max(1, min(n, _SLAB_BYTES // (n * n * 16)))


def _write_npy_header(f, n):
    np.lib.format.write_array_header_1_0(f, dict(_NPY_C128, shape=(n, n, n)))


def _read_npy_header(f):
    major, minor = np.lib.format.read_magic(f)
    reader = {(1, 0): np.lib.format.read_array_header_1_0,
              (2, 0): np.lib.format.read_array_header_2_0}.get((major, minor))
    if reader is None:
        raise ValueError(f"unsupported .npy version {major}.{minor}")
    return reader(f)


def save_wavefunction(path, stage, step):
    """Write ``stage.psi`` (complex64 or complex128, on any device) as a complex128
    snapshot with its metadata and axes."""
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    psi = stage.psi
    n = int(stage.N_grids)
    per = _planes_per_slab(n)
    with open(path, "wb") as f:
        _write_npy_header(f, n)
        if not psi.is_cuda:
            for x0 in range(0, n, per):
                f.write(psi[x0:x0 + per].to(torch.complex128).contiguous().numpy().tobytes())
        else:
            dev = psi.device
            copy = torch.cuda.Stream(dev)
            wide = torch.empty((per, n, n), dtype=torch.complex128, device=dev)
            pinned = [torch.empty((per, n, n), dtype=torch.complex128).pin_memory() for _ in range(2)]
            landed = [torch.cuda.Event() for _ in range(2)]
            pending = []   # (buffer index, planes) copied but not yet written
            copy.wait_stream(torch.cuda.current_stream(dev))
            for s, x0 in enumerate(range(0, n, per)):
                b, rows = s % 2, min(per, n - x0)
                if len(pending) == 2:        # buffer b still holds slab s-2: write it first
                    ob, orows = pending.pop(0)
                    landed[ob].synchronize()
                    f.write(pinned[ob][:orows].numpy().tobytes())
                with torch.cuda.stream(copy):
                    wide[:rows].copy_(psi[x0:x0 + rows])                 # widen on the device
                    pinned[b][:rows].copy_(wide[:rows], non_blocking=True)
                    landed[b].record(copy)
                pending.append((b, rows))
            for ob, orows in pending:
                landed[ob].synchronize()
                f.write(pinned[ob][:orows].numpy().tobytes())
    np.savez(path.parent / "grid.npz", x_array=_host(stage.x_array), k_array=_host(stage.k_array))
    meta = {"step": step, "time": step * stage.dt, "evolution": stage.type, "N_atom": stage.N_atoms,
            "simulation_range": stage.simulation_range, "N_grids": n, "stage": getattr(stage, "config", {})}
    path.with_suffix(".json").write_text(json.dumps(meta, indent=2) + "\n")


def _check_companions(path, stage):
    """The metadata and axes beside a snapshot, where present, must describe this
    stage's box, reference atom number and grid."""
    meta_path = path.with_suffix(".json")
    if meta_path.exists():
        meta = json.loads(meta_path.read_text())
        if meta["simulation_range"] != stage.simulation_range:
            raise ValueError(f"{path.name} was saved for simulation_range {meta['simulation_range']}, "
                             f"not {stage.simulation_range}")
        if meta["N_atom"] != stage.N_atoms:
            raise ValueError(f"{path.name} was saved for N_atom {meta['N_atom']}, not {stage.N_atoms}")
    for grid_path in (path.with_name(path.stem + "_grid.npz"), path.parent / "grid.npz"):
        if grid_path.exists():
            with np.load(grid_path, allow_pickle=False) as grid:
                for name in ("x_array", "k_array"):
                    want = _host(getattr(stage, name))
                    have = grid[name]
                    if have.shape != want.shape or not np.allclose(have, want):
                        raise ValueError(f"{grid_path.name}: {name} differs from this stage's grid")
            break


def load_wavefunction(path, stage, dtype=torch.complex128):
    """A saved complex128 cube for ``stage``, as ``dtype`` on the stage's device;
    its norm and clock are left as they are."""
    path = Path(path)
    n = int(stage.N_grids)
    with open(path, "rb") as f:
        head = _read_npy_header(f)
        shape, fortran, descr = head
        if tuple(shape) != (n, n, n) or fortran or np.dtype(descr) != np.complex128:
            raise ValueError(f"{path.name} holds {np.dtype(descr)} {tuple(shape)}"
                             f"{' (Fortran order)' if fortran else ''}; this stage needs a complex128 "
                             f"C-order cube of {n}^3")
        _check_companions(path, stage)
        device = stage.x_array.device if isinstance(stage.x_array, torch.Tensor) else torch.device("cpu")
        psi = torch.empty((n, n, n), dtype=dtype, device=device)
        per = _planes_per_slab(n)
        plane = n * n * 16
        if device.type != "cuda":
            for x0 in range(0, n, per):
                rows = min(per, n - x0)
                raw = np.frombuffer(f.read(rows * plane), dtype=np.complex128).reshape(rows, n, n)
                psi[x0:x0 + rows] = torch.from_numpy(raw.copy()).to(dtype)
            return psi
        copy = torch.cuda.Stream(device)
        wide = [torch.empty((per, n, n), dtype=torch.complex128, device=device) for _ in range(2)]
        pinned = [torch.empty((per, n, n), dtype=torch.complex128).pin_memory() for _ in range(2)]
        free = [None, None]   # events: the copy out of pinned buffer b has finished
        with torch.cuda.stream(copy):
            for s, x0 in enumerate(range(0, n, per)):
                b, rows = s % 2, min(per, n - x0)
                if free[b] is not None:
                    free[b].synchronize()                    # buffer b's previous slab has left
                got = f.readinto(memoryview(pinned[b].numpy()[:rows]).cast("B"))
                if got != rows * plane:
                    raise ValueError(f"{path.name} ends before its {n}^3 cube does")
                wide[b][:rows].copy_(pinned[b][:rows], non_blocking=True)
                free[b] = torch.cuda.Event()
                free[b].record(copy)
                psi[x0:x0 + rows].copy_(wide[b][:rows])     # narrow on the device
        torch.cuda.current_stream(device).wait_stream(copy)
        return psi
