"""GPU edge cases: the smallest systems against closed forms (the reference's
one- and two-atom checks), a 40-site fixed-excitation sector through the
64-bit generic kernel, and one-state sectors."""
import numpy as np
import pytest

from oracle import ref
from energy_level_b200 import configs

pytestmark = pytest.mark.gpu
CONV = 2 * np.pi * 1e-3


def one_atom_calib():
    return {"atoms": [{"id": 0, "pos": [0.0, 0.0, 0.0]}], "pairs": [], "terms": ["I1"]}


@pytest.mark.parametrize("Delta", [0.0, 1.3])
def test_single_atom_rabi_closed_form(ctx, Delta):
    """P_r(t) = Om^2 / (Om^2 + Delta^2) sin^2(sqrt(Om^2 + Delta^2) CONV t / 2)."""
    from energy_level_b200.engine import evolve_manybody
    Om = 2.0
    t = np.linspace(0.0, 800.0, 9)
    r = evolve_manybody(one_atom_calib(), "g", t, Om=np.array([Om]), delta=np.array([-Delta]))
    W = np.sqrt(Om ** 2 + Delta ** 2)
    want = Om ** 2 / W ** 2 * np.sin(W * CONV * t / 2) ** 2
    assert np.abs(r["pops_atom"][:, 0] - want).max() < 1e-10
    assert np.abs(r["norms"] - 1.0).max() < 1e-12


def test_blockaded_pair_collective_rabi(ctx):
    """Two atoms in perfect blockade: |gg> oscillates with sqrt(2) Om."""
    from energy_level_b200.engine import evolve_manybody
    calib = {"atoms": [{"id": 0, "pos": [0.0, 0.0, 0.0]}, {"id": 1, "pos": [2.0, 0.0, 0.0]}],
             "pairs": [], "terms": ["I1"]}
    plan = {"projected": True, "blockade_edges": [[0, 1]], "constraint": {"kind": "blockade"}}
    Om = 1.5
    t = np.linspace(0.0, 600.0, 7)
    r = evolve_manybody(calib, "gg", t, Om=np.full(2, Om), delta=np.zeros(2), plan=plan, record_psi=True)
    assert r["basis"]["dim"] == 3
    p_gg = np.cos(np.sqrt(2) * Om * CONV * t[-1] / 2) ** 2
    assert abs(abs(r["psi_amp"][0]) ** 2 - p_gg) < 1e-10
    want_each = 0.5 * np.sin(np.sqrt(2) * Om * CONV * t / 2) ** 2
    assert np.abs(r["pops_atom"] - want_each[:, None]).max() < 1e-10


def test_forty_site_sector_generic_kernel(ctx):
    """n = 40 (64-bit codes, generic kernel), two excitations, XY exchange."""
    import torch
    from energy_level_b200 import solvers
    from energy_level_b200.core import Basis, Hamiltonian
    n, k = 40, 2
    xy = configs.xy_chain(n, seed=9)
    pairs = [(p["i"], p["j"], p["V"]) for p in xy["calib"]["pairs"]]
    ex = [(p["i"], p["j"], p["J"], 0.0) for p in xy["calib"]["pairs"]]
    b = Basis(ctx, n, kind="charge", k=k)
    codes = ref.number_sector_basis(n, k)
    assert b.dim == len(codes) == n * (n - 1) // 2
    assert np.array_equal(b.codes().cpu().numpy(), codes)
    h = Hamiltonian(ctx, b, np.zeros(n), xy["delta"], pairs, exchange=ex)
    rng = np.random.default_rng(5)
    x = rng.normal(size=b.dim)
    y = h.hv(torch.as_tensor(x, dtype=torch.float64, device=ctx.device)).cpu().numpy()
    want = ref.hv(n, codes, np.zeros(n), xy["delta"], pairs, x, exchange=ex)
    assert np.abs(y - want).max() < 1e-12 * max(1.0, np.abs(want).max())
    r = solvers.lanczos_ground(h, dtype="float64", tol=1e-11, nev=2, max_iter=400)
    w = np.linalg.eigvalsh(ref.dense_h(n, codes, np.zeros(n), xy["delta"], pairs, exchange=ex))
    assert r["converged"] and abs(r["evals"][0] - w[0]) < 1e-9


def test_one_state_sectors(ctx):
    """k = 0 and k = n sectors hold one state: E0 is its diagonal entry."""
    from energy_level_b200 import solvers
    from energy_level_b200.core import Basis, Hamiltonian
    n = 8
    xy = configs.xy_chain(n, seed=1)
    pairs = [(p["i"], p["j"], p["V"]) for p in xy["calib"]["pairs"]]
    ex = [(p["i"], p["j"], p["J"], 0.0) for p in xy["calib"]["pairs"]]
    for k in (0, n):
        b = Basis(ctx, n, kind="charge", k=k)
        assert b.dim == 1
        h = Hamiltonian(ctx, b, np.zeros(n), xy["delta"], pairs, exchange=ex)
        r = solvers.lanczos_ground(h, dtype="float64", tol=1e-12, nev=2, max_iter=10)
        d = ref.diagonal(n, ref.number_sector_basis(n, k), xy["delta"], pairs)[0]
        assert r["converged"] and abs(r["evals"][0] - d) < 1e-12


def test_constraint_plans_match_reference_ground_states(ctx):
    """Bases and ground states of plans given only as constraint specs
    (threshold edges on a 3x4 lattice: a general blockade graph in the table
    layout; 'auto' pxp; mode='full') against the reference's build_plan
    states and ground_state energies."""
    import json
    import os
    from energy_level_b200 import model, solvers
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "constraint.npz"))
    calib = configs.calib_from_positions(g["pos"])
    for nm in g["names"]:
        nm = str(nm)
        spec = json.loads(str(g[nm + "_spec"]))
        projected = bool(g[nm + "_projected"])
        plan = {"projected": projected, "constraint": spec, "calib": calib}
        _, basis, ham, _ = model.build(calib, g["om"], g["de"], plan=plan if projected else None,
                                       constraint=spec)
        assert basis.dim == int(g[nm + "_dim"]), nm
        if projected:
            assert np.array_equal(basis.codes().cpu().numpy(), g[nm + "_states"]), nm
        r = solvers.lanczos_ground(ham, dtype="float64", tol=1e-12, nev=2, max_iter=min(400, basis.dim))
        assert r["converged"], nm
        assert abs(r["evals"][0] - float(g[nm + "_E0"])) < 1e-9, nm
        assert abs((r["evals"][1] - r["evals"][0]) - float(g[nm + "_gap"])) < 1e-7, nm
