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


def _due_steps(stage):
    save = getattr(stage, "save_params", None) or {}
    monitor = getattr(stage, "monitor_params", None) or {}
    scalar = [save.get("scalar_interval"), monitor.get("print_scalar_interval")]
    spectrum = [save.get("nk_interval"), monitor.get("show_nk_interval")]
    return scalar, spectrum


def launch_stage(stage, on_diagnostics=None):
    """Run a prepared stage and return its final wavefunction (``stage.psi``)."""
    scalar, spectrum = _due_steps(stage)
    intervals = [i for i in scalar + spectrum if i]
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
