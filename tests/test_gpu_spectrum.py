"""Source-state spectrum on the GPU against the reference's fixture
(tests/golden/spectrum.npz): device Lanczos tridiagonal, broadened spectrum
and the want='spectrum' route."""
import os

import numpy as np
import pytest

from energy_level_b200 import configs

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(__file__), "golden", "spectrum.npz")


def _ham(ctx, g):
    from energy_level_b200.core import Basis, Hamiltonian
    n = int(g["n"])
    b = Basis(ctx, n, kind="blockade", edges=configs.chain_edges(n))
    assert np.array_equal(b.codes().cpu().numpy(), g["codes"])
    pairs = [(int(a), int(c), float(v)) for a, c, v in g["pairs"]]
    return Hamiltonian(ctx, b, g["om"], g["de"], pairs)


@pytest.mark.parametrize("dtype,tol", [("complex128", 1e-9), ("complex64", 2e-4)])
def test_device_lanczos_matches_reference(ctx, dtype, tol):
    from energy_level_b200 import spectrum as spec
    g = np.load(G)
    h = _ham(ctx, g)
    lz = spec.lanczos(h, g["phi"], 40, dtype=dtype)
    assert lz["n"] == int(g["lz_n"]) and lz["reortho"]
    assert abs(lz["norm2"] - float(g["norm2"])) < (1e-12 if dtype == "complex128" else 1e-6)
    scale = np.max(np.abs(g["alphas"]))
    assert np.max(np.abs(lz["alphas"] - g["alphas"])) < tol * scale
    assert np.max(np.abs(lz["betas"] - g["betas"])) < tol * scale
    assert lz["ortho_loss"] < 1e-6 if dtype == "complex128" else lz["ortho_loss"] < 1e-3


def test_source_spectrum_matches_reference(ctx):
    from energy_level_b200 import spectrum as spec
    g = np.load(G)
    h = _ham(ctx, g)
    out = spec.source_spectrum(h, g["phi"], shift=0.3, eta=0.1, n_krylov=40, n_omega=300)
    assert np.allclose(out["omega"], g["sp_omega"], atol=1e-10)
    assert np.max(np.abs(out["spectral"] - g["sp_spectral"])) < 1e-8 * max(1.0, np.abs(g["sp_spectral"]).max())
    assert np.allclose(out["evals"], g["sp_evals"], atol=1e-8)
    for key in ("omega", "spectral", "evals", "spectrum_weights", "source_norm", "eta", "shift", "krylov",
                "error_report"):
        assert key in out


def test_spectrum_route_matches_reference(ctx):
    from energy_level_b200.backends import solve_equilibrium
    g = np.load(G)
    n = int(g["n"])
    calib = configs.calib_from_positions(configs.chain_positions(n))
    system = {"calib": calib, "Om": g["om"], "delta": g["de"], "terms": ["I1"],
              "source": {"kind": "site_weights", "weights": g["weights"], "subtract_mean": True},
              "spectrum": {"eta": 0.1, "n_krylov": 40, "n_omega": 300}}
    r = solve_equilibrium(system, want="spectrum", backend="b200-lanczos")
    assert abs(r["E0"] - float(g["route_E0"])) < 1e-8
    assert abs(r["source_norm"] - float(g["route_source_norm"])) < 1e-8
    # the window comes from the extreme Ritz values of a 40-step run, which
    # move with the last digits of |0>; compare the spectra on one grid
    assert np.allclose(r["energies"][[0, -1]], g["route_energies"][[0, -1]], atol=1e-3)
    ours = np.interp(g["route_energies"], r["energies"], r["spectral"])
    scale = np.abs(g["route_spectral"]).max()
    assert np.max(np.abs(ours - g["route_spectral"])) < 2e-3 * scale, np.max(np.abs(ours - g["route_spectral"]))
    assert r["gap"] is None and r["error_report"]["source_kind"] == "site_weights"
