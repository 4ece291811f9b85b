"""Stage time loop (``gpe/launch.py:4-14``).

The reference calls the per-step closure once per step from Python and runs
``save_outputs`` after each.  Here the steps between two due diagnostic
points run as one multi-step C-ABI call (``closure.run``), with the same
time convention ``t = i*dt`` for step ``i``; at due steps the fused
diagnostics (N, E_kin, E, mu and optionally n(k)) of the completed state are
recorded.
"""

import csv
from pathlib import Path

import numpy as np

from .helper import is_due


# monitor interval -> image outputs it asks for (gpe/save.py:59-90)
_IMAGES = {"show_TOF_image_interval": ("TOF_xy",), "show_verticle_TOF_interval": ("TOF_yz",),
           "show_TOF_slice_interval": ("TOF_slice_xy",), "show_verticle_TOF_slice_interval": ("TOF_slice_yz",),
           "show_magnifier_interval": ("density_xy",), "show_magnifier_slice_interval": ("density_slice_xy",),
           "show_phase_interval": ("phase_xy",)}


def _due_steps(stage):
    save = getattr(stage, "save_params", None) or {}
    monitor = getattr(stage, "monitor_params", None) or {}
    scalar = [save.get("scalar_interval"), monitor.get("print_scalar_interval")]
    spectrum = [save.get("nk_interval"), monitor.get("show_nk_interval")]
    images = {key: monitor.get(key) for key in _IMAGES}
    images["psi_interval"] = save.get("psi_interval")
    return scalar, spectrum, images


def _snapshot(stage, step):
    """``psi_<step>.npy`` in the stage's data folder (``gpe/save.py:15-17``)."""
    from .state_io import save_wavefunction
    folder = getattr(stage, "data_dir", None)
    if folder is not None:
        save_wavefunction(Path(folder) / f"psi_{step:08d}.npy", stage, step)


def launch_stage(stage, on_diagnostics=None):
    """Run a prepared stage and return its final wavefunction (``stage.psi``)."""
    scalar, spectrum, images = _due_steps(stage)
    save = getattr(stage, "save_params", None) or {}
    if save.get("save_initial"):
        _snapshot(stage, 0)
    intervals = [i for i in scalar + spectrum + list(images.values()) if i]
    prop = stage.propagator
    history = []
    i = 0
    while i < stage.steps:
        stop = stage.steps
        for iv in intervals:
            nxt = (i // iv + 1) * iv
            stop = min(stop, nxt)
        if hasattr(prop, "run"):
            prop.run(stage, stop - i, i)
        else:
            for j in range(i, stop):
                stage.psi = prop(stage, j * stage.dt) if getattr(prop, "dynamic", False) else prop(stage)
        i = stop
        want_scalar = any(is_due(i, iv) for iv in scalar)
        want_nk = any(is_due(i, iv) for iv in spectrum)
        want_img = [name for key, iv in images.items() if key in _IMAGES and is_due(i, iv)
                    for name in _IMAGES[key]]
        if is_due(i, images["psi_interval"]) or (i == stage.steps and save.get("save_final")):
            _snapshot(stage, i)
        if want_img:
            plan, psi = prop.binding.plan(stage)
            _write_images(stage, i, plan.projections(psi, want_img))
        if want_scalar or want_nk:
            plan, psi = prop.binding.plan(stage)
            rec = plan.diagnostics(psi, t=i * stage.dt, nk=want_nk)
            if want_scalar:
                rec["Lz"] = plan.angular_momentum(psi)
            rec.update(step=i, time=i * stage.dt)
            history.append(rec)
            _write(stage, rec, want_scalar, want_nk)
            if on_diagnostics:
                on_diagnostics(stage, rec)
    stage.history = history
    return stage.psi


def _write_images(stage, step, images):
    """The reference's image files (``gpe/save.py:59-90``): ``<name>_<step>.npz``
    with ``step``, ``time``, ``values`` and the axes."""
    folder = getattr(stage, "monitor_dir", None)
    if folder is None:
        return
    folder = Path(folder)
    folder.mkdir(parents=True, exist_ok=True)
    x = stage.x_array.detach().cpu().numpy() if hasattr(stage.x_array, "detach") else np.asarray(stage.x_array)
    k = stage.k_array.detach().cpu().numpy() if hasattr(stage.k_array, "detach") else np.asarray(stage.k_array)
    ks = np.fft.fftshift(k)
    mid = stage.N_grids // 2
    axes = {"TOF_xy": dict(kx=ks, ky=ks), "TOF_yz": dict(ky=ks, kz=ks), "TOF_slice_xy": dict(kx=ks, ky=ks),
            "TOF_slice_yz": dict(ky=ks, kz=ks), "density_xy": dict(x=x, y=x),
            "density_slice_xy": dict(x=x, y=x, z=x[mid]), "phase_xy": dict(x=x, y=x, z=x[mid])}
    for name, values in images.items():
        np.savez(folder / f"{name}_{step:08d}.npz", step=step, time=step * stage.dt, values=values, **axes[name])


def _write(stage, rec, scalar, nk):
    folder = getattr(stage, "monitor_dir", None)
    if folder is None:
        return
    folder = Path(folder)
    folder.mkdir(parents=True, exist_ok=True)
    if scalar:
        path = folder / "scalars.csv"
        new = not path.exists()
        with path.open("a", newline="") as f:
            w = csv.writer(f)
            if new:
                # the reference's columns (gpe/save.py:53), then total energy and mu
                w.writerow(["step", "time", "norm", "N_atoms", "E_kin", "Lz", "E", "mu"])
            w.writerow([rec["step"], rec["time"], rec["N"], stage.N_atoms * rec["N"], rec["E_kin"],
                        rec["Lz"], rec["E"], rec["mu"]])
    if nk:
        np.savez(folder / f"nk_{rec['step']:08d}.npz", step=rec["step"], time=rec["time"],
                 Nk=rec["Nk"], counts=rec["counts"])
