"""The register-resident sweeps (n = 32 ... 256) against the generic
mixed-radix sweeps and the oracle, for every step sequence they implement."""

import numpy as np
import pytest
import torch

from oracle import ssf
from tests.golden import cases

pytestmark = pytest.mark.gpu


def make(n, L, kind, dtype, generic, **kw):
    from gpe_simulator_b200 import Plan
    x, k = ssf.get_grids(n, L)
    return Plan(n, x, k, dtype=dtype, kind=kind, generic_only=generic, **kw), x


@pytest.mark.parametrize("n", [32, 48, 64, 96, 128, 160])
@pytest.mark.parametrize("dtype,tol", [(torch.complex128, 1e-13), (torch.complex64, 3e-6)])
@pytest.mark.parametrize("kind", ["imaginary", "real"])
def test_fast_matches_generic_and_oracle(cuda, n, dtype, tol, kind):
    from gpe_simulator_b200 import Beam
    kw = dict(beta=800.0, dt=4e-4, static_expr=cases.TRAP)
    if kind == "real":
        kw["beam"] = Beam(20.0, 0.5, 2.0, 1.0, 0.004)
    fast, x = make(n, 12.0, kind, dtype, False, **kw)
    slow, _ = make(n, 12.0, kind, dtype, True, **kw)
    psi0 = ssf.noisy_gaussian(x, seed=n)
    a = torch.from_numpy(psi0).to(dtype).cuda()
    b = a.clone()
    fast.step(a, 7, 3)
    slow.step(b, 7, 3)
    err = ssf.rel_l2(a.cpu().numpy(), b.cpu().numpy())
    assert err < tol, err
    m = ssf.Model(n=n, simulation_range=12.0, kind=kind, beta=800.0, dt=4e-4, static_expr=cases.TRAP,
                  beam=ssf.Beam(20.0, 0.5, 2.0, 1.0, 0.004) if kind == "real" else None)
    want = ssf.run(psi0, m, 7, step0=3)
    err = ssf.rel_l2(a.cpu().numpy(), want)
    assert err < (1e-12 if dtype == torch.complex128 else 1e-5), err


@pytest.mark.parametrize("n", [32, 48, 64, 96, 128, 160, 256])
@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
@pytest.mark.parametrize("kind", ["imaginary", "real"])
def test_fast_diagnostics_match_generic_and_oracle(cuda, n, dtype, kind):
    """Diagnostics on the register-resident sweeps (z: real-space sums and the
    forward transform; y; x: forward transform, sum k^2 |psi_k|^2 and the shell
    histogram) against the generic sweeps and the oracle on the same state at a
    time where the beam has moved.  Both paths agree to 1e-12 on the sums of
    psi itself (N, E_pot, E_int); against the oracle, complex64 E_pot carries
    the FP32 evaluation of the potential (1e-8) and E_kin and n(k) the FP32
    transform's rounding."""
    from gpe_simulator_b200 import Beam
    kw = dict(beta=800.0, dt=4e-4, static_expr=cases.TRAP)
    if kind == "real":
        kw["beam"] = Beam(20.0, 0.5, 2.0, 1.0, 0.004)
    fast, x = make(n, 12.0, kind, dtype, False, **kw)
    slow, _ = make(n, 12.0, kind, dtype, True, **kw)
    psi = torch.from_numpy(ssf.noisy_gaussian(x, seed=n)).to(dtype).cuda()
    t = 0.003
    a, b = fast.diagnostics(psi, t=t, nk=True), slow.diagnostics(psi, t=t, nk=True)
    c128 = dtype == torch.complex128
    m = ssf.Model(n=n, simulation_range=12.0, kind=kind, beta=800.0, dt=4e-4, static_expr=cases.TRAP,
                  beam=ssf.Beam(20.0, 0.5, 2.0, 1.0, 0.004) if kind == "real" else None)
    state = psi.cpu().numpy()
    want = ssf.energies(state, m, t=t)
    spec = ssf.nk_extraction(np.fft.fftn(state.astype(np.complex128)), x, m.k)
    for key in ("N", "E_pot", "E_int", "E_kin", "E", "mu"):
        same = 1e-12 if (c128 or key in ("N", "E_pot", "E_int")) else 1e-6
        assert a[key] == pytest.approx(b[key], rel=same), (key, a[key], b[key])
        oracle = 1e-12 if (c128 or key in ("N", "E_int")) else (1e-7 if key == "E_pot" else 1e-6)
        assert a[key] == pytest.approx(want[key], rel=oracle), (key, a[key], want[key])
    np.testing.assert_array_equal(a["counts"], spec["counts"])
    np.testing.assert_allclose(a["Nk"], spec["Nk"], rtol=1e-10 if c128 else 1e-5,
                               atol=(1e-14 if c128 else 1e-8) * spec["Nk"].max())
    # energies alone (no shell histogram) give the same sums
    e = fast.diagnostics(psi, t=t)
    assert all(e[key] == a[key] for key in ("N", "E_kin", "E_pot", "E_int"))
    assert fast.status() == 0


@pytest.mark.parametrize("n", [32, 48, 64, 96, 128, 160, 256])
def test_fast_fft_matches_numpy(cuda, n):
    p, _ = make(n, 10.0, "imaginary", torch.complex64, False, beta=0.0, dt=0.0)
    g = torch.Generator(device="cuda").manual_seed(n)
    a = torch.randn((n, n, n), dtype=torch.complex64, device="cuda", generator=g)
    f = p.fft(a)
    ref = torch.fft.fftn(a.to(torch.complex128))
    err = ((f.to(torch.complex128) - ref).abs().pow(2).sum() / ref.abs().pow(2).sum()).sqrt().item()
    assert err < 2e-6, err
    back = p.fft(f, inverse=True)
    err = ((back - a).abs().pow(2).sum() / a.abs().pow(2).sum()).sqrt().item()
    assert err < 2e-6, err


def test_step_at_equals_step(cuda):
    """``propagator(stage, t)`` one call at a time equals one multi-step call."""
    from gpe_simulator_b200 import Beam
    p, x = make(64, 12.0, "real", torch.complex128, False, beta=500.0, dt=5e-4,
                static_expr=cases.TRAP, beam=Beam(20.0, 0.5, 2.0, 1.0, 0.002))
    a = torch.from_numpy(ssf.noisy_gaussian(x, seed=1)).cuda()
    b = a.clone()
    p.step(a, 6, 0)
    for i in range(6):
        p.step_at(b, i * 5e-4)
    assert ssf.rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 1e-14


@pytest.mark.parametrize("n", [128, 256])
@pytest.mark.parametrize("kind", ["imaginary", "real"])
def test_plane_fused_equals_unfused_bitwise(cuda, n, kind):
    """The plane-fused launches (y and z sweeps of an x-plane in one launch) run
    exactly the per-tile arithmetic of the separate sweeps: identical bits."""
    from gpe_simulator_b200 import Beam
    kw = dict(beta=800.0, dt=4e-4, static_expr=cases.TRAP)
    if kind == "real":
        kw["beam"] = Beam(20.0, 0.5, 2.0, 1.0, 0.004)
    fused, x = make(n, 12.0, kind, torch.complex64, False, fuse_planes=True, **kw)
    plain, _ = make(n, 12.0, kind, torch.complex64, False, **kw)
    a = torch.from_numpy(ssf.noisy_gaussian(x, seed=n)).to(torch.complex64).cuda()
    b = a.clone()
    for s0, k in ((0, 5), (5, 1), (6, 4)):
        fused.step(a, k, s0)
        plain.step(b, k, s0)
    assert torch.equal(a, b)
    assert fused.status() == 0 and plain.status() == 0


@pytest.mark.parametrize("n", [128, 256])
@pytest.mark.parametrize("kind", ["imaginary", "real"])
def test_tma_staged_sweeps_equal_plain_loads_bitwise(cuda, n, kind):
    """The y/x sweeps whose pencils arrive by TMA (persistent, double-buffered)
    run the arithmetic of the register-resident sweeps with plain loads:
    identical bits for step sequences, out-of-place transforms (x sweeps, source
    != destination), and a state whose address is not 16-byte aligned (staging
    is skipped there)."""
    from gpe_simulator_b200 import Beam
    kw = dict(beta=800.0, dt=4e-4, static_expr=cases.TRAP)
    if kind == "real":
        kw["beam"] = Beam(20.0, 0.5, 2.0, 1.0, 0.004)
    staged, x = make(n, 12.0, kind, torch.complex64, False, tma=True, **kw)
    plain, _ = make(n, 12.0, kind, torch.complex64, False, **kw)
    a = torch.from_numpy(ssf.noisy_gaussian(x, seed=n + 1)).to(torch.complex64).cuda()
    b = a.clone()
    for s0, k in ((0, 5), (5, 1), (6, 4)):
        staged.step(a, k, s0)
        plain.step(b, k, s0)
    assert torch.equal(a, b)
    fa, fb = staged.fft(a), plain.fft(b)
    assert torch.equal(fa, fb)
    assert torch.equal(staged.fft(fa, inverse=True), plain.fft(fb, inverse=True))
    # an 8-byte offset view: the tensor map would not be 16-byte aligned
    buf = torch.zeros(n ** 3 + 1, dtype=torch.complex64, device="cuda")
    c = buf[1:].view(n, n, n)
    c.copy_(a)
    staged.step(c, 3, 10)
    plain.step(b, 3, 10)
    assert torch.equal(c, b)
    assert staged.status() == 0 and plain.status() == 0


def test_auto_path_is_timed_cached_and_bit_identical(cuda, tmp_path, monkeypatch):
    """``Plan(path="auto")`` times the three complex64 sweep paths at 128^3 once,
    caches the fastest, and computes the same bits as the default path."""
    import json
    from gpe_simulator_b200 import Beam, tune
    monkeypatch.setenv("GPE_TUNE_CACHE", str(tmp_path / "paths.json"))
    kw = dict(beta=800.0, dt=4e-4, static_expr=cases.TRAP, beam=Beam(20.0, 0.5, 2.0, 1.0, 0.004))
    auto, x = make(128, 12.0, "real", torch.complex64, False, path="auto", **kw)
    plain, _ = make(128, 12.0, "real", torch.complex64, False, **kw)
    assert auto.path in tune.CANDIDATES and plain.path == "default"
    cache = json.loads((tmp_path / "paths.json").read_text())
    (entry,) = cache.values()
    assert entry["path"] == auto.path
    assert all(v > 0 for v in entry["ms_per_step"].values())
    assert entry["ms_per_step"][auto.path] == min(entry["ms_per_step"].values())
    a = torch.from_numpy(ssf.noisy_gaussian(x, seed=5)).to(torch.complex64).cuda()
    b = a.clone()
    auto.step(a, 6, 0)
    plain.step(b, 6, 0)
    assert torch.equal(a, b)


@pytest.mark.parametrize("kind", ["imaginary", "real"])
def test_fast_512_matches_generic(cuda, kind):
    """512^3 complex64 (the largest single solve): register-resident sweeps vs
    the generic mixed-radix sweeps (the latter checked against the oracle at
    smaller sizes), a few steps."""
    from gpe_simulator_b200 import Beam
    kw = dict(beta=2000.0, dt=1.25e-4, static_expr=cases.TRAP)
    if kind == "real":
        kw["beam"] = Beam(20.0, 0.5, 2.0, 1.0, 0.025)
    fast, x = make(512, 24.0, kind, torch.complex64, False, **kw)
    slow, _ = make(512, 24.0, kind, torch.complex64, True, **kw)
    g = np.exp(-x ** 2 / 2)
    a = (torch.from_numpy(g).cuda()[:, None, None] * torch.from_numpy(g).cuda()[None, :, None]
         * torch.from_numpy(g).cuda()[None, None, :]).to(torch.complex64)
    a = a * (1 + 0.01 * torch.randn(a.shape, dtype=torch.complex64, device="cuda",
                                    generator=torch.Generator(device="cuda").manual_seed(5)))
    fast.normalise(a)
    b = a.clone()
    fast.step(a, 4, 0)
    slow.step(b, 4, 0)
    err = (((a - b).abs() ** 2).sum() / (b.abs() ** 2).sum()).sqrt().item()
    assert err < 3e-6, err


@pytest.mark.parametrize("kind", ["imaginary", "real"])
def test_local_fp64_plans_run_the_fp64_local_factor(cuda, kind):
    """local_fp64 (complex64 plans: local factor in FP64) runs on the generic
    sweeps, which carry that variant: same bits as a generic-only plan, and
    different arithmetic from the FP32 default."""
    from gpe_simulator_b200 import Beam
    kw = dict(beta=800.0, dt=4e-4, static_expr=cases.TRAP, local_fp64=True)
    if kind == "real":
        kw["beam"] = Beam(20.0, 0.5, 2.0, 1.0, 0.004)
    lf, x = make(64, 12.0, kind, torch.complex64, False, **kw)
    gen, _ = make(64, 12.0, kind, torch.complex64, True, **kw)
    plain, _ = make(64, 12.0, kind, torch.complex64, False, **{**kw, "local_fp64": False})
    a = torch.from_numpy(ssf.noisy_gaussian(x, seed=4)).to(torch.complex64).cuda()
    b, c = a.clone(), a.clone()
    lf.step(a, 7, 3)
    gen.step(b, 7, 3)
    plain.step(c, 7, 3)
    assert torch.equal(a, b)
    assert not torch.equal(a, c)
    assert ssf.rel_l2(a.cpu().numpy(), c.cpu().numpy()) < 3e-6
