"""GPU parity of the device observables (el_spin_observables, el_pauli_expect)
and of the evolution's observable contract, against golden vectors written
by the reference and against the oracle."""
import os

import numpy as np
import pytest

from oracle import ref
from energy_level_b200 import configs

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def gold():
    return np.load(os.path.join(GOLD, "observables.npz"))


def _ham(ctx, n, codes_kind):
    from energy_level_b200.core import Basis, Hamiltonian
    if codes_kind == "full":
        b = Basis(ctx, n, kind="full")
    else:
        b = Basis(ctx, n, kind="blockade", edges=configs.chain_edges(n))
    return b, Hamiltonian(ctx, b, np.zeros(n), np.zeros(n), [])


def _matrices(ob, n, pairs):
    NN = np.diag(ob["n"]).astype(float)
    XY = np.diag(ob["n"]).astype(complex)
    for q, (i, j) in enumerate(pairs):
        NN[i, j] = ob["nn"][q]
        XY[i, j] = ob["xy"][q]
    return NN, XY


@pytest.mark.parametrize("which", ["full", "basis"])
@pytest.mark.parametrize("dtype", ["complex128", "complex64"])
def test_spin_observables_match_reference(ctx, which, dtype):
    import torch
    from energy_level_b200 import solvers
    g = gold()
    n = 7 if which == "full" else 10
    b, h = _ham(ctx, n, which)
    if which == "basis":
        assert np.array_equal(b.codes().cpu().numpy(), g["basis_states"])
    psi = torch.as_tensor(g[which + "_psi"], dtype=getattr(torch, dtype), device=ctx.device)
    pairs = [(i, j) for i in range(n) for j in range(n) if i != j]
    ob = solvers.spin_observables(h, psi, pairs)
    tol = 1e-12 if dtype == "complex128" else 2e-6
    sm = ob["sm"]
    assert np.abs(2 * sm.real - g[which + "_sx"]).max() < tol
    assert np.abs(2 * sm.imag - g[which + "_sy"]).max() < tol
    assert np.abs(ob["norm"] - 2 * ob["n"] - g[which + "_sz"]).max() < tol
    assert np.abs(sm - g[which + "_sm"]).max() < tol
    NN, XY = _matrices(ob, n, pairs)
    assert np.abs(XY - g[which + "_xy_corr"]).max() < tol
    if which == "basis":
        corr = NN - np.outer(ob["n"], ob["n"])
        assert np.abs(corr - g["basis_corr"]).max() < tol


@pytest.mark.parametrize("which", ["full", "basis"])
def test_pauli_strings_match_oracle(ctx, which):
    import torch
    from energy_level_b200 import solvers
    g = gold()
    n = 7 if which == "full" else 10
    b, h = _ham(ctx, n, which)
    codes = None if which == "full" else g["basis_states"]
    v = g[which + "_psi"]
    specs = [{"label": "a", "terms": [(0, "x")]}, {"label": "b", "terms": [(1, "y"), (3, "z")]},
             {"label": "c", "terms": [(2, "x"), (4, "y"), (5, "z"), (6, "x")]},
             {"label": "d", "terms": [(6, "z"), (0, "y")]}, {"label": "e", "terms": [(1, "y"), (2, "y")]}]
    want = np.asarray([ref.pauli_expect(n, codes, v, sp["terms"]) for sp in specs])
    for dt, tol in (("complex128", 1e-12), ("complex64", 2e-6)):
        psi = torch.as_tensor(v, dtype=getattr(torch, dt), device=ctx.device)
        got = solvers.pauli_expect(h, psi, specs)
        assert np.abs(got - want).max() < tol, dt


def test_pauli_and_pair_refusals(ctx):
    import torch
    from energy_level_b200 import solvers
    _, h = _ham(ctx, 6, "full")
    psi = torch.ones(64, dtype=torch.complex128, device=ctx.device)
    with pytest.raises(ValueError):
        solvers.pauli_expect(h, psi, [{"label": "x", "terms": [(0, "x"), (0, "z")]}])
    with pytest.raises(ValueError):
        solvers.pauli_expect(h, psi, [{"label": "x", "terms": [(7, "x")]}])
    with pytest.raises(ValueError):
        solvers.spin_observables(h, psi, [(2, 2)])


def test_schmidt_entropy_matches_reference(ctx):
    import torch
    from energy_level_b200.engine import _Schmidt
    g = gold()
    b, _ = _ham(ctx, 7, "full")
    s = _Schmidt(b, 7, 3, ctx.device)
    psi = torch.as_tensor(g["full_psi"], dtype=torch.complex128, device=ctx.device)
    assert abs(s.entropy(psi) - float(g["full_S3"])) < 1e-12
    b, _ = _ham(ctx, 10, "basis")
    s = _Schmidt(b, 10, 5, ctx.device)
    psi = torch.as_tensor(g["basis_psi"], dtype=torch.complex128, device=ctx.device)
    assert abs(s.entropy(psi) - float(g["basis_S5"])) < 1e-12


def _segments(g, tag, n):
    return [{"t0": float(t0), "Om": om, "delta": de}
            for t0, om, de in zip(g[tag + "_seg_t0"], g[tag + "_seg_om"], g[tag + "_seg_de"])]


def _check_evolution(r, g, tag, keys_obs, tol=1e-8):
    for k in ("pops_atom", "corr", "norms", "pops", "basis_probabilities"):
        assert np.abs(np.asarray(r[k]) - g[tag + "_" + k]).max() < tol, k
    assert np.allclose(r["S"], g[tag + "_S"], atol=tol, rtol=0, equal_nan=True)
    assert np.abs(r["psi_amp"] - g[tag + "_psi_amp"]).max() < tol
    for k in keys_obs:
        want = g[tag + "_obs_" + k]
        got = np.asarray(r["observables"][k])
        if k == "phase":
            assert np.allclose(got, want, atol=1e-6, rtol=0, equal_nan=True)
        else:
            assert np.abs(got - want).max() < tol, k


def test_evolution_observables_full_basis_match_reference(ctx):
    """XY exchange + drive, three segments, link correlations."""
    from energy_level_b200.engine import evolve_manybody
    g = gold()
    n = int(g["ev1_n"])
    xy = configs.xy_chain(n, seed=21)
    r = evolve_manybody(xy["calib"], "rg" * (n // 2), g["ev1_t"], segments=_segments(g, "ev1", n),
                        terms=["I1", "I2"], record_psi=True, link_pairs=[(0, 1), (2, 4)])
    _check_evolution(r, g, "ev1", ("sx", "sy", "sz", "sp", "sm", "phase", "xy_corr", "link_corr"))
    assert len(r["states"]) == 1 << n and r["states"][5]["label"] == "|gggrgr>"
    assert r["error_report"]["full_pops"]


def test_evolution_observables_projected_match_reference(ctx):
    from energy_level_b200.engine import evolve_manybody
    g = gold()
    n = int(g["ev2_n"])
    calib = configs.calib_from_positions(configs.chain_positions(n))
    plan = {"projected": True, "blockade_edges": configs.chain_edges(n), "states": g["ev2_states"],
            "constraint": {"kind": "blockade"}}
    r = evolve_manybody(calib, "g" * n, g["ev2_t"], segments=_segments(g, "ev2", n), plan=plan,
                        terms=["I1"], record_psi=True)
    assert np.array_equal(r["basis_states"], g["ev2_states"])
    _check_evolution(r, g, "ev2", ("sx", "sy", "sz", "sp", "sm", "phase", "xy_corr"))


def test_evolution_pauli_strings_and_loops(ctx):
    from energy_level_b200.engine import evolve_manybody
    from energy_level_b200.observables import loop_observables
    n = 6
    xy = configs.xy_chain(n, seed=4)
    specs = [[[0, "x"], [1, "y"]], {"label": "zz", "terms": [[2, "z"], [3, "z"]]}]
    t = np.linspace(0.0, 200.0, 3)
    r = evolve_manybody(xy["calib"], "rg" * 3, t, Om=np.full(n, 0.7), delta=xy["delta"], terms=["I1", "I2"],
                        record_psi=True, pauli_strings=specs, loops=[[0, 1, 2]],
                        link_pairs=[(0, 1), (1, 2), (2, 0)])
    ob = r["observables"]
    assert ob["pauli_string_labels"] == ["x@0 y@1", "zz"]
    for q, terms in enumerate([[(0, "x"), (1, "y")], [(2, "z"), (3, "z")]]):
        assert abs(ob["pauli_strings"][-1, q] - ref.pauli_expect(n, None, r["psi_amp"], terms)) < 1e-10
    ph, wd = loop_observables(ob["xy_corr"], [[0, 1, 2]])
    assert np.allclose(ob["loop_phase"], ph, equal_nan=True) and np.allclose(ob["loop_winding"], wd, equal_nan=True)
    assert ob["loop_phase_series"].shape == (3, 1)
    assert np.allclose(ob["loop_phase_series"][-1, 0], ph[0], atol=1e-9, equal_nan=True)
    with pytest.raises(ValueError):
        evolve_manybody(xy["calib"], "rg" * 3, t, Om=np.full(n, 0.7), terms=["I1", "I2"],
                        pauli_strings=specs, want_observables=False)
    with pytest.raises(ValueError):
        evolve_manybody(xy["calib"], "rg" * 3, t, Om=np.full(n, 0.7), terms=["I1", "I2"],
                        link_pairs=[(0, 9)])


@pytest.mark.parametrize("kind", ["charge", "ring"])
def test_spin_observables_other_layouts_match_oracle(ctx, kind):
    """Fixed-excitation (table-ranked) and ring sectors against the oracle."""
    import torch
    from energy_level_b200 import solvers
    from energy_level_b200.core import Basis, Hamiltonian
    n = 10
    if kind == "charge":
        b = Basis(ctx, n, kind="charge", k=4)
        codes = ref.number_sector_basis(n, 4)
    else:
        b = Basis(ctx, n, kind="blockade", edges=configs.ring_edges(n))
        codes = ref.independent_states(n, configs.ring_edges(n), None)
    h = Hamiltonian(ctx, b, np.zeros(n), np.zeros(n), [])
    rng = np.random.default_rng(8)
    v = rng.normal(size=b.dim) + 1j * rng.normal(size=b.dim)
    v /= np.linalg.norm(v)
    want = ref.spin_observables(n, codes, v)
    pairs = [(i, j) for i in range(n) for j in range(n) if i != j]
    ob = solvers.spin_observables(h, torch.as_tensor(v, dtype=torch.complex128, device=ctx.device), pairs)
    assert np.abs(ob["sm"] - want["sm"]).max() < 1e-12
    _, XY = _matrices(ob, n, pairs)
    assert np.abs(XY - want["xy_corr"]).max() < 1e-12
