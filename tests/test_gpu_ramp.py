"""Equilibrium ramp (warm-started ground states along (Omega_t, delta_t)) on
the GPU against the reference's want='ramp' fixture (tests/golden/ramp.npz)."""
import os

import numpy as np
import pytest

from energy_level_b200 import configs

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(__file__), "golden", "ramp.npz")


@pytest.mark.parametrize("warm", [True, False])
def test_ramp_matches_reference(ctx, warm):
    from energy_level_b200.backends import solve_equilibrium
    g = np.load(G)
    n = int(g["n"])
    calib = configs.calib_from_positions(configs.chain_positions(n))
    n_tot = np.asarray([bin(c).count("1") for c in range(1 << n)], float)
    r = solve_equilibrium({"calib": calib, "terms": ["I1"]}, want="ramp", backend="b200-lanczos",
                          ramp={"Om_t": g["Om_t"], "de_t": g["de_t"], "L": n, "n_tot": n_tot,
                                "v0_warm": warm})
    assert np.allclose(r["taus"], g["taus"])
    assert r["converged"].all()
    assert np.max(np.abs(r["gaps"] - g["gaps"])) < 1e-7
    assert np.max(np.abs(r["ns"] - g["ns"])) < 1e-8


def test_ramp_needs_calib_and_L(ctx):
    from energy_level_b200.backends import solve_equilibrium
    calib = configs.calib_from_positions(configs.chain_positions(4))
    with pytest.raises(ValueError):
        solve_equilibrium({"calib": calib}, want="ramp", backend="b200-lanczos",
                          ramp={"Om_t": [1.0], "de_t": [0.0]})
    with pytest.raises(ValueError):
        solve_equilibrium({"n_sites": 4}, want="ramp", backend="b200-lanczos",
                          ramp={"Om_t": [1.0], "de_t": [0.0], "L": 4})
