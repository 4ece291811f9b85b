"""Snapshots in the reference's format (``gpe/state_io.py``): round trips across
precisions, the reference's checks, the files the reference's own
``save_wavefunction`` wrote (``tests/golden/state_ref``, made by
``tests/golden/make_state_files.py``), and a live exchange with the reference's
save/load run on the host through the oracle shim where GPE_REFERENCE is set."""

import json
from pathlib import Path

from types import SimpleNamespace

import numpy as np
import pytest
import torch

from gpe_simulator_b200.state_io import load_wavefunction, save_wavefunction

from oracle import ref_shim  # noqa: E402

STATE_REF = Path(__file__).resolve().parent / "golden" / "state_ref"


def make_stage(n=8, L=6.0, dtype=torch.complex64, seed=0):
    x = torch.linspace(-L / 2, L / 2 - L / n, n, dtype=torch.float64)
    k = torch.from_numpy(2 * np.pi * np.fft.fftfreq(n, L / n))
    g = torch.Generator().manual_seed(seed)
    psi = torch.randn((n, n, n), dtype=torch.complex128, generator=g).to(dtype)
    return SimpleNamespace(psi=psi, x_array=x, k_array=k, N_grids=n, dt=0.01, type="real", N_atoms=1000,
                           simulation_range=L, config={"name": "test"})


@pytest.mark.parametrize("dtype", [torch.complex64, torch.complex128])
def test_round_trip_through_complex128_file(tmp_path, dtype):
    st = make_stage(dtype=dtype)
    save_wavefunction(tmp_path / "psi_00000007.npy", st, 7)
    saved = np.load(tmp_path / "psi_00000007.npy")
    assert saved.dtype == np.complex128 and saved.shape == (8, 8, 8)
    np.testing.assert_array_equal(saved, st.psi.to(torch.complex128).numpy())
    back = load_wavefunction(tmp_path / "psi_00000007.npy", st, dtype)
    assert back.dtype == dtype and torch.equal(back, st.psi)
    meta = (tmp_path / "psi_00000007.json").read_text()
    assert '"step": 7' in meta and '"N_atom": 1000' in meta
    assert (tmp_path / "grid.npz").exists()


def test_load_rejects_what_the_reference_rejects(tmp_path):
    st = make_stage()
    save_wavefunction(tmp_path / "a.npy", st, 0)
    with pytest.raises(ValueError):
        load_wavefunction(tmp_path / "a.npy", make_stage(n=10))
    other = make_stage()
    other.N_atoms = 5
    with pytest.raises(ValueError):
        load_wavefunction(tmp_path / "a.npy", other)
    other = make_stage(L=7.0)
    with pytest.raises(ValueError):
        load_wavefunction(tmp_path / "a.npy", other)
    np.save(tmp_path / "b.npy", np.zeros((8, 8, 8), np.complex64))
    with pytest.raises(ValueError):
        load_wavefunction(tmp_path / "b.npy", st)


def test_files_written_by_the_reference_load_and_match_ours_byte_for_byte(tmp_path):
    """The reference's snapshot of the seeded stage loads in both precisions; our
    save of the same stage gives the same .npy bytes, metadata and axes."""
    st = make_stage(dtype=torch.complex128)
    for dtype in (torch.complex128, torch.complex64):
        back = load_wavefunction(STATE_REF / "psi_00000004.npy", st, dtype)
        assert back.dtype == dtype and torch.equal(back, st.psi.to(dtype))
    save_wavefunction(tmp_path / "psi_00000004.npy", st, 4)
    assert (tmp_path / "psi_00000004.npy").read_bytes() == (STATE_REF / "psi_00000004.npy").read_bytes()
    assert (json.loads((tmp_path / "psi_00000004.json").read_text())
            == json.loads((STATE_REF / "psi_00000004.json").read_text()))
    with np.load(tmp_path / "grid.npz") as ours, np.load(STATE_REF / "grid.npz") as theirs:
        assert sorted(ours.files) == sorted(theirs.files) == ["k_array", "x_array"]
        for name in ours.files:
            np.testing.assert_array_equal(ours[name], theirs[name])


@pytest.mark.skipif(not ref_shim.available(), reason=ref_shim.UNSET if ref_shim.REFERENCE is None
                    else "no reference sources where GPE_REFERENCE points")
def test_files_exchange_with_the_reference(tmp_path):
    ref = ref_shim.install()
    st = make_stage(dtype=torch.complex128)
    save_wavefunction(tmp_path / "ours" / "psi.npy", st, 3)
    rst = SimpleNamespace(N_grids=8, simulation_range=st.simulation_range, N_atoms=st.N_atoms,
                          x_array=st.x_array.numpy(), k_array=st.k_array.numpy(), psi=st.psi.numpy(),
                          dt=st.dt, type="real", config={})
    np.testing.assert_array_equal(ref.state_io.load_wavefunction(tmp_path / "ours" / "psi.npy", rst),
                                  st.psi.numpy())
    ref.state_io.save_wavefunction(tmp_path / "theirs" / "psi.npy", rst, 4)
    assert torch.equal(load_wavefunction(tmp_path / "theirs" / "psi.npy", st), st.psi)
