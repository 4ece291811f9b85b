"""Generate the golden fixtures from the reference implementation itself.

Runs ONLY where ``GPE_REFERENCE`` names the reference's source tree.  The
reference's own ``gpe`` package is imported with a
NumPy-backed CuPy (``oracle/ref_shim.py``): its propagator closures
(``gpe/make_propagator.py``), its CUDA kernel strings compiled for the host
(``gpe/kernels.py``, ``gpe/make_kernel.py``, ``gpe/helper.py``) and its
diagnostics (``gpe/helper.py:135-140``, ``gpe/nk_extraction.py:16-45``) produce
every number stored here; only cuFFT is replaced by numpy.fft.

All cases are in reference units (kinetic factor ``exp(-i k^2 dt)``).  Inputs
are regenerated from the stored seeds, so the fixtures hold outputs only:

* ``ground64``   config "plain imaginary-time ground state": N=64, box
  [-8,8)^3, V = x^2+1.44y^2+2.25z^2 (= 2 x the oscillator-unit trap),
  beta = 1000 (g = 500), dt = 5e-4 (oscillator dt = 1e-3), seeded noisy
  Gaussian (seed 0), 2000 steps; checkpoints at 100, 1000, 2000.
* ``stir32``     200 imaginary steps from a noisy Gaussian (seed 1), then 400
  real-time steps with the harmonic trap plus a rotating Gaussian beam written
  in the reference's expression grammar.  N=32, box [-12,12)^3, beta = 2000.
* ``lossy16``    real time with a complex static potential (absorber ``-i
  Gamma`` ramp plus a real box) and a momentum cutoff, N=16.
* ``box24``      imaginary time with a float64 box potential array plus a
  static expression, N=24.
* ``diag_n*``    ``get_N``, ``get_E``, ``get_L`` and ``nk_extraction`` of seeded states.
* ``proj_n*``    the image outputs of ``save_outputs`` (TOF columns and slices, column
                 density, density slice and phase) of seeded states.

Usage: ``python tests/golden/make_golden.py`` (writes ``tests/golden/*.npz``).
"""

import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import ref_shim, ssf  # noqa: E402
from tests.golden import cases  # noqa: E402

OUT = Path(__file__).resolve().parent


def summary(psi, x, k, ref, sub):
    """Subsampled field, random projections and reference diagnostics of psi."""
    psi = np.ascontiguousarray(psi)
    out = dict(psi_sub=psi[::sub, ::sub, ::sub].copy(),
               proj=cases.projections(psi),
               N=float(ref.helper.get_N(psi, x)),
               E_kin=float(ref.helper.get_E(np.fft.fftn(psi), x, k)))
    return out


def save(name, **arrays):
    np.savez_compressed(OUT / f"{name}.npz", **arrays)
    print("wrote", name, flush=True)


def make_ground64(ref):
    c = cases.GROUND64
    st = ref_shim.reference_stage(ref, n=c["n"], simulation_range=c["L"], kind="imaginary",
                                  beta=c["beta"], dt=c["dt"], static_expr=c["static_expr"])
    psi = ssf.noisy_gaussian(st.x_array, seed=c["seed"])
    out, done = {}, 0
    for mark in c["checkpoints"]:
        t0 = time.time()
        psi = ref_shim.run_reference(ref, st, psi, mark - done, step0=done)
        done = mark
        for key, val in summary(psi, st.x_array, st.k_array, ref, c["sub"]).items():
            out[f"{key}_{mark}"] = val
        print(f"ground64 step {mark} ({time.time() - t0:.0f}s)", flush=True)
    save("ground64", **out)


def make_stir32(ref):
    c = cases.STIR32
    imag = ref_shim.reference_stage(ref, n=c["n"], simulation_range=c["L"], kind="imaginary",
                                    beta=c["beta"], dt=c["dt"], static_expr=c["static_expr"])
    psi = ssf.noisy_gaussian(imag.x_array, seed=c["seed"])
    psi = ref_shim.run_reference(ref, imag, psi, c["imag_steps"])
    start = summary(psi, imag.x_array, imag.k_array, ref, c["sub"])
    real = ref_shim.reference_stage(ref, n=c["n"], simulation_range=c["L"], kind="real",
                                    beta=c["beta"], dt=c["dt"], static_expr=c["static_expr"],
                                    dynamic_expr=cases.stir_beam().expression())
    out = {"psi_start": start["psi_sub"], "N_start": start["N"]}
    done = 0
    for mark in c["checkpoints"]:
        psi = ref_shim.run_reference(ref, real, psi, mark - done, step0=done)
        done = mark
        for key, val in summary(psi, real.x_array, real.k_array, ref, c["sub"]).items():
            out[f"{key}_{mark}"] = val
    save("stir32", **out)


def make_lossy16(ref):
    c = cases.LOSSY16
    x, _ = ssf.get_grids(c["n"], c["L"])
    st = ref_shim.reference_stage(ref, n=c["n"], simulation_range=c["L"], kind="real",
                                  beta=c["beta"], dt=c["dt"], static_expr=c["static_expr"],
                                  dynamic_expr=c["dynamic_expr"], k_cut=c["k_cut"],
                                  static_v=cases.lossy_potential(x, c))
    psi = ssf.noisy_gaussian(x, sigma=1.5, seed=c["seed"])
    psi = ref_shim.run_reference(ref, st, psi, c["steps"])
    save("lossy16", psi=psi, N=float(ref.helper.get_N(psi, st.x_array)))


def make_box24(ref):
    c = cases.BOX24
    x, _ = ssf.get_grids(c["n"], c["L"])
    st = ref_shim.reference_stage(ref, n=c["n"], simulation_range=c["L"], kind="imaginary",
                                  beta=c["beta"], dt=c["dt"], static_expr=c["static_expr"],
                                  static_v=cases.box_potential(x, c))
    psi = ssf.noisy_gaussian(x, sigma=2.0, seed=c["seed"])
    psi = ref_shim.run_reference(ref, st, psi, c["steps"])
    save("box24", psi=psi)


def make_diag(ref):
    for n, L in cases.DIAG_SIZES:
        x, k = ref.grids.get_grids(n, L)
        psi = cases.diag_state(n)
        F = np.fft.fftn(psi)
        spec = ref.nk_extraction.nk_extraction(F, x, k, slab_size=3)
        save(f"diag_n{n}", N=float(ref.helper.get_N(psi, x)),
             E_kin=float(ref.helper.get_E(F, x, k)), L=float(ref.helper.get_L(psi, x, k, slab_size=3)),
             **{f"nk_{key}": np.asarray(val) for key, val in spec.items()})


def make_proj(ref):
    """The reference's own save_outputs (``gpe/save.py:59-90``) with every image
    output due, on seeded states (even and odd n: fftshift)."""
    import tempfile
    from types import SimpleNamespace
    for n, L in cases.PROJ_SIZES:
        x, k = ref.grids.get_grids(n, L)
        psi = cases.diag_state(n, seed=7)
        with tempfile.TemporaryDirectory() as tmp:
            monitor = {name: 1 for name in ("show_TOF_image_interval", "show_verticle_TOF_interval",
                                            "show_TOF_slice_interval", "show_verticle_TOF_slice_interval",
                                            "show_magnifier_interval", "show_magnifier_slice_interval",
                                            "show_phase_interval")}
            monitor.update(print_scalar_interval=None, show_nk_interval=None)
            st = SimpleNamespace(save_params=dict(psi_interval=None, save_initial=False, save_final=False,
                                                  scalar_interval=None, nk_interval=None),
                                 monitor_params=monitor, monitor_dir=Path(tmp), psi=psi, x_array=x,
                                 k_array=k, N_grids=n, dt=0.1, name="proj")
            ref.save.save_outputs(st, 1)
            files = {"TOF_xy": "TOF_xy", "TOF_yz": "TOF_yz", "TOF_slice_xy": "TOF_slice_xy",
                     "TOF_slice_yz": "TOF_slice_yz", "density_xy": "density_xy",
                     "density_slice_xy": "density_slice_xy", "phase_xy": "phase_xy"}
            vals = {key: np.load(Path(tmp) / f"{name}_00000001.npz")["values"] for key, name in files.items()}
        save(f"proj_n{n}", **vals)


def main(which=None):
    ref = ref_shim.install()
    jobs = dict(diag=make_diag, proj=make_proj, lossy16=make_lossy16, box24=make_box24,
                stir32=make_stir32, ground64=make_ground64)
    for name, job in jobs.items():
        if which is None or name in which:
            job(ref)


if __name__ == "__main__":
    main(sys.argv[1:] or None)
