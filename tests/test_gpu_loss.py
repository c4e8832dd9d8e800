"""GPU parity of the loss (non-Hermitian gamma) path: H x with the loss
diagonal, the Taylor propagator and evolve_manybody with gamma, against
golden vectors written by the reference and against the oracle."""
import os

import numpy as np
import pytest

from oracle import ref
from energy_level_b200 import configs

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def gold():
    return np.load(os.path.join(GOLD, "loss.npz"))


@pytest.mark.parametrize("name", ["full7", "chain10"])
def test_loss_hv_matches_reference(ctx, name):
    import torch
    from energy_level_b200.core import Basis, Hamiltonian
    g = gold()
    n = 7 if name == "full7" else 10
    calib = configs.calib_from_positions(configs.chain_positions(n))
    pairs = [(p["i"], p["j"], p["V"]) for p in calib["pairs"]]
    b = Basis(ctx, n, kind="full") if name == "full7" else Basis(ctx, n, kind="blockade",
                                                                   edges=configs.chain_edges(n))
    p = "hv_" + name + "_"
    h = Hamiltonian(ctx, b, g[p + "om"], g[p + "de"], pairs)
    h.set_loss(g[p + "ga"])
    assert h.lossy and h.complex_drive
    want = g[p + "y"]
    for dt, tol in (("complex128", 1e-12), ("complex64", 2e-5)):
        x = torch.as_tensor(g[p + "x"], dtype=getattr(torch, dt), device=ctx.device)
        got = h.hv(x).cpu().numpy()
        assert np.abs(got - want).max() <= tol * max(1.0, np.abs(want).max()), dt
    with pytest.raises(ValueError):
        h.hv(torch.ones(b.dim, dtype=torch.float64, device=ctx.device))
    h.set_loss(None)
    assert not h.lossy


def test_taylor_step_matches_chebyshev_when_hermitian(ctx):
    import torch
    from energy_level_b200 import solvers
    from energy_level_b200.core import Basis, Hamiltonian
    n = 12
    calib = configs.calib_from_positions(configs.chain_positions(n))
    pairs = [(p["i"], p["j"], p["V"]) for p in calib["pairs"]]
    b = Basis(ctx, n, kind="blockade", edges=configs.chain_edges(n))
    h = Hamiltonian(ctx, b, np.full(n, 2.0), np.full(n, -1.0), pairs)
    rng = np.random.default_rng(2)
    v = rng.normal(size=b.dim) + 1j * rng.normal(size=b.dim)
    v /= np.linalg.norm(v)
    a = torch.as_tensor(v, dtype=torch.complex128, device=ctx.device)
    c = a.clone()
    nt = solvers.taylor_step(h, a, 137.0, tol=1e-13)
    solvers.cheb_step(h, c, 137.0, tol=1e-13)
    assert nt > 0
    assert float((a - c).abs().max()) < 1e-11


def test_lossy_refusals(ctx):
    import torch
    from energy_level_b200 import solvers
    from energy_level_b200.core import Basis, Hamiltonian
    from energy_level_b200.matrix_free import b200_lanczos_ground_state
    from energy_level_b200.model import ConfigConflict
    n = 6
    b = Basis(ctx, n, kind="full")
    h = Hamiltonian(ctx, b, np.ones(n), np.zeros(n), [])
    h.set_loss(np.full(n, 1.0))
    psi = torch.zeros(1 << n, dtype=torch.complex128, device=ctx.device)
    psi[0] = 1
    with pytest.raises(ValueError):
        solvers.cheb_step(h, psi, 10.0)
    with pytest.raises(ValueError):
        solvers.lanczos_ground(h, dtype="complex128")
    calib = configs.calib_from_positions(configs.chain_positions(n))
    with pytest.raises(ConfigConflict):
        b200_lanczos_ground_state(calib, np.ones(n), np.zeros(n), gamma=np.full(n, 1.0))


def test_loss_evolution_full_basis_matches_reference(ctx):
    from energy_level_b200.engine import evolve_manybody
    g = gold()
    n = 6
    xy = configs.xy_chain(n, seed=31)
    segs = [{"t0": float(t0), "Om": om, "delta": de}
            for t0, om, de in zip(g["ev1_seg_t0"], g["ev1_seg_om"], g["ev1_seg_de"])]
    for dt, tol in (("complex128", 1e-9), ("complex64", 2e-5)):
        r = evolve_manybody(xy["calib"], "rg" * 3, g["ev1_t"], segments=segs, gamma=g["ev1_ga"],
                            terms=["I1", "I2"], record_psi=True, dtype=dt)
        assert r["backend"] == "b200-cheb-nonhermitian" and not r["error_report"]["hermitian"]
        for k in ("pops_atom", "norms", "loss", "corr"):
            assert np.abs(np.asarray(r[k]) - g["ev1_" + k]).max() < tol, (dt, k)
        assert np.allclose(r["S"], g["ev1_S"], atol=tol * 10, rtol=0, equal_nan=True)
        assert np.abs(r["psi_amp"] - g["ev1_psi_amp"]).max() < tol, dt


def test_loss_evolution_projected_matches_reference(ctx):
    from energy_level_b200.engine import evolve_manybody
    g = gold()
    n = 9
    calib = configs.calib_from_positions(configs.chain_positions(n))
    plan = {"projected": True, "blockade_edges": configs.chain_edges(n), "states": g["ev2_states"],
            "constraint": {"kind": "blockade"}}
    r = evolve_manybody(calib, "g" * n, g["ev2_t"], Om=np.full(n, 2.0), delta=np.full(n, -1.0),
                        gamma=g["ev2_ga"], plan=plan, terms=["I1"], record_psi=True)
    for k in ("pops_atom", "norms", "loss", "corr"):
        assert np.abs(np.asarray(r[k]) - g["ev2_" + k]).max() < 1e-9, k
    assert np.allclose(r["S"], g["ev2_S"], atol=1e-8, rtol=0, equal_nan=True)
    assert np.abs(r["psi_amp"] - g["ev2_psi_amp"]).max() < 1e-9
    # the oracle agrees as well
    pairs = [(p["i"], p["j"], p["V"]) for p in calib["pairs"]]
    psi0 = np.zeros(len(g["ev2_states"]), complex)
    psi0[0] = 1.0
    seg = [{"t0": 0.0, "Om": np.full(n, 2.0), "delta": np.full(n, -1.0)}]
    want = ref.evolve_segments(n, g["ev2_states"], pairs, seg, psi0, g["ev2_t"], gamma=g["ev2_ga"])
    assert np.abs(r["psi_amp"] - want[-1]).max() < 1e-9
