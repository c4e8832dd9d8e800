"""Source-state spectrum: oracle Lanczos and host post-processing against the
reference's fixture (tests/golden/spectrum.npz)."""
import os

import numpy as np

from oracle import ref

G = os.path.join(os.path.dirname(__file__), "golden", "spectrum.npz")


def _g():
    return np.load(G)


def test_oracle_lanczos_matches_reference():
    g = _g()
    n = int(g["n"])
    codes = g["codes"]
    pairs = [(int(a), int(b), float(v)) for a, b, v in g["pairs"]]
    al, be, k = ref.lanczos_tridiag(lambda v: ref.hv(n, codes, g["om"], g["de"], pairs, v),
                                    g["phi"], 40)
    assert k == int(g["lz_n"])
    assert np.max(np.abs(al - g["alphas"])) < 1e-9
    assert np.max(np.abs(be - g["betas"])) < 1e-9


def test_host_quadrature_and_lorentz_match_reference():
    from energy_level_b200 import spectrum as spec
    g = _g()
    norm2 = float(g["norm2"])
    nodes, w = spec.quadrature(g["alphas"], g["betas"], norm2, 0.3)
    assert np.allclose(nodes, g["sp_evals"], atol=1e-10)
    assert np.allclose(w, g["sp_weights"], atol=1e-12)
    s = spec.lorentz_spectrum(g["alphas"], g["betas"], norm2, g["sp_omega"], 0.1, 0.3)
    assert np.max(np.abs(s - g["sp_spectral"])) < 1e-10


def test_resolve_source_kinds():
    from energy_level_b200 import spectrum as spec
    n = 4
    codes = ref.independent_states(n, [[0, 1], [1, 2], [2, 3]], None)
    rng = np.random.default_rng(0)
    psi = rng.normal(size=len(codes)) + 0j
    psi /= np.linalg.norm(psi)
    w = np.array([1.0, -1.0, 0.5, 0.0])
    phi, info = spec.resolve_source({"kind": "site_weights", "weights": w, "subtract_mean": True},
                                    psi, n, codes)
    bits = ref.basis_bits(n, codes).astype(float)
    d = bits.T @ w
    mean = np.vdot(psi, d * psi).real
    assert np.allclose(phi, (d - mean) * psi) and abs(info["subtracted_mean"] - mean) < 1e-14
    phi2, _ = spec.resolve_source({"kind": "psi0"}, psi, n, codes)
    assert np.allclose(phi2, psi)
    import pytest
    with pytest.raises(ValueError):
        spec.resolve_source({"kind": "vector", "values": [1.0]}, psi, n, codes)
    with pytest.raises(ValueError):
        spec.resolve_source({"kind": "bogus"}, psi, n, codes)
