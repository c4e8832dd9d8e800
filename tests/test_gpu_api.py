"""GPU tests of the reference-facing API against golden vectors written by
the reference itself (tests/golden)."""
import os

import numpy as np
import pytest

from energy_level_b200 import configs

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def gold(name):
    return np.load(os.path.join(GOLD, name + ".npz"))


def calib_of(pairs, n):
    return {"atoms": [{"id": i, "pos": [float(i), 0.0, 0.0]} for i in range(n)],
            "pairs": [{"i": int(i), "j": int(j), "V": float(v), "J": 0.0, "A": 0.0} for i, j, v in pairs],
            "terms": ["I1"]}


def plan_of(n, edges, codes=None):
    return {"projected": True, "blockade_edges": [list(e) for e in edges], "states": codes,
            "constraint": {"kind": "blockade"}}


def test_ground_state_chain12_full_and_blockade(ctx):
    from energy_level_b200.matrix_free import b200_lanczos_ground_state
    g = gold("ground")
    cfg = configs.chain12()
    r = b200_lanczos_ground_state(cfg["calib"], cfg["Om"], cfg["delta"], tol=1e-12, m=400)
    assert r["converged"] and r["backend"] == "b200-lanczos" and r["dim"] == 4096
    assert abs(r["E0"] - float(g["chain12_E0"])) < 1e-9
    assert abs(r["gap"] - float(g["chain12_gap"])) < 1e-8
    for key in ("E0", "gap", "evals", "residuals", "converged", "backend", "dim", "krylov_dim",
                "restarts", "tolerance"):
        assert key in r
    rb = b200_lanczos_ground_state(cfg["calib"], cfg["Om"], cfg["delta"], tol=1e-12,
                                   plan=plan_of(12, configs.chain_edges(12)), return_state=True)
    assert abs(rb["E0"] - float(g["chain12b_E0"])) < 1e-9
    assert abs(np.linalg.norm(rb["vec"]) - 1.0) < 1e-9
    r32 = b200_lanczos_ground_state(cfg["calib"], cfg["Om"], cfg["delta"], dtype="float32")
    assert r32["converged"] and abs(r32["E0"] - float(g["chain12_E0"])) < 1e-6 * abs(float(g["chain12_E0"]))


def test_ground_state_ring20_blockade(ctx):
    from energy_level_b200.matrix_free import b200_lanczos_ground_state
    g = gold("ground")
    calib = calib_of(g["ring20_pairs"], 20)
    r = b200_lanczos_ground_state(calib, np.full(20, 2.0), np.full(20, 1.0), tol=1e-10,
                                  plan=plan_of(20, configs.ring_edges(20)))
    assert r["dim"] == 15127 and r["converged"]
    assert abs(r["E0"] - float(g["ring20_E0"])) < 1e-8


def test_unsorted_basis_indices_roundtrip(ctx):
    """basis_indices in any order (channels selfcheck semantics): the state
    comes back in the caller's order."""
    from energy_level_b200.matrix_free import b200_lanczos_ground_state
    from oracle import ref
    n = 8
    calib = configs.calib_from_positions(configs.chain_positions(n))
    codes = ref.independent_states(n, configs.chain_edges(n), None)
    perm = np.random.default_rng(0).permutation(len(codes))
    r1 = b200_lanczos_ground_state(calib, np.full(n, 1.3), np.full(n, -0.5), basis_indices=codes,
                                   return_state=True, tol=1e-11)
    r2 = b200_lanczos_ground_state(calib, np.full(n, 1.3), np.full(n, -0.5), basis_indices=codes[perm],
                                   return_state=True, tol=1e-11)
    assert abs(r1["E0"] - r2["E0"]) < 1e-10
    v1, v2 = r1["vec"][perm], r2["vec"]
    assert abs(abs(np.vdot(v1, v2)) - 1.0) < 1e-9
    with pytest.raises(ValueError):
        b200_lanczos_ground_state(calib, np.full(n, 1.3), np.zeros(n), basis_indices=[0, 0, 1])


@pytest.mark.parametrize("name", ["full7", "chain10", "ring9", "square3x3", "cplx8"])
def test_operator_matches_reference_matvec(ctx, name):
    from energy_level_b200.matrix_free import hamiltonian_operator
    g = gold("hv")
    n = int(g["n_" + name])
    edges = g["edges_" + name].tolist()
    calib = calib_of(g["pairs_" + name], n)
    plan = plan_of(n, edges) if edges else None
    op = hamiltonian_operator(calib, g["om_" + name], g["de_" + name], plan=plan)
    y = op @ g["x_" + name]
    assert np.max(np.abs(y - g["y_" + name])) < 1e-12 * max(1.0, np.abs(g["y_" + name]).max())


@pytest.mark.parametrize("mode", ["direct", "doubling"])
def test_kpm_with_reference_probes_matches_reference(ctx, mode):
    from energy_level_b200.kpm import kpm_moments_b200
    g = gold("kpm")
    n = int(g["n"])
    system = {"calib": calib_of(g["pairs"], n), "Om": g["om"], "delta": g["de"]}
    mu, c, r = kpm_moments_b200(system, num=int(g["num"]), nvec=int(g["nvec"]), dtype="float64",
                                probes=g["probes"], bounds=(float(g["emin"]), float(g["emax"])), mode=mode,
                                chunk=4)
    assert abs(c - float(g["c"])) < 1e-12 and abs(r - float(g["r"])) < 1e-12
    assert np.max(np.abs(mu - g["mu"])) < 1e-10
    mu2, c2, r2, info = kpm_moments_b200(system, num=int(g["num"]), nvec=int(g["nvec"]), dtype="float64",
                                         probes=g["probes"], return_info=True, chunk=4)
    assert abs(info["emin"] - float(g["emin"])) < 1e-8 and abs(info["emax"] - float(g["emax"])) < 1e-8
    assert np.max(np.abs(mu2 - g["mu"])) < 1e-7


@pytest.mark.parametrize("dtype,tol", [("complex128", 1e-9), ("complex64", 2e-5)])
def test_evolution_matches_reference(ctx, dtype, tol):
    from energy_level_b200.engine import evolve_manybody
    g = gold("evolve")
    n = int(g["n"])
    calib = calib_of(g["pairs"], n)
    segs = [{"t0": float(t), "Om": om, "delta": de} for t, om, de in zip(g["seg_t0"], g["seg_om"], g["seg_de"])]
    res = evolve_manybody(calib, psi0="g" * n, t_grid=g["t_grid"], segments=segs,
                          plan=plan_of(n, configs.chain_edges(n)), record_psi=True, dtype=dtype)
    assert np.array_equal(res["basis_states"], g["basis_states"])
    assert np.max(np.abs(res["psi_amp"] - g["psi_final"])) < tol
    assert np.max(np.abs(res["pops_atom"] - g["pops_atom"])) < tol
    assert np.max(np.abs(res["norms"] - 1.0)) < tol
    for key in ("t", "pops", "states", "method", "backend", "pops_atom", "S", "corr", "loss", "norms",
                "basis_states", "basis", "error_report"):
        assert key in res


def test_cancel_flag_stops_evolution(ctx):
    from energy_level_b200.engine import evolve_manybody
    n = 6
    calib = configs.calib_from_positions(configs.chain_positions(n))
    prog = np.array([0.0, 1.0])
    with pytest.raises(RuntimeError, match="用户取消"):
        evolve_manybody(calib, psi0="g" * n, t_grid=[0.0, 10.0], Om=np.ones(n), delta=np.zeros(n),
                        progress_arr=prog)


def test_solve_equilibrium_routes(ctx):
    from energy_level_b200.backends import solve_equilibrium
    g = gold("ground")
    cfg = configs.chain12()
    sysd = {"calib": cfg["calib"], "Om": cfg["Om"], "delta": cfg["delta"],
            "plan": dict(plan_of(12, configs.chain_edges(12)), states=None)}
    r = solve_equilibrium(sysd, "gs", backend="b200-lanczos")
    assert abs(r["E0"] - float(g["chain12b_E0"])) < 1e-8 and r["n_atom"].shape == (12,)
    d = solve_equilibrium({"calib": cfg["calib"], "Om": cfg["Om"], "delta": cfg["delta"]}, "dos",
                          backend="b200-kpm", num=64, nvec=8)
    assert d["rho"].shape == (400,) and np.all(d["rho"] >= 0)
    t = solve_equilibrium({"calib": cfg["calib"], "Om": cfg["Om"], "delta": cfg["delta"]}, "thermal",
                          backend="b200-kpm", betas=[0.1], num=128, nvec=16)
    assert np.isfinite(t["E"]).all()


def test_batched_ground_states_match_dense(ctx):
    """Uneven chain/ring sectors in one persistent launch vs dense eigh."""
    from energy_level_b200.batched import batched_ground_states
    from oracle import ref
    rng = np.random.default_rng(4)
    insts, want = [], []
    for k in range(24):
        n = int(rng.integers(6, 13))
        ring = (k % 3 == 0)
        edges = configs.ring_edges(n) if ring else configs.chain_edges(n)
        calib = configs.calib_from_positions(configs.chain_positions(n, jitter=rng.uniform(-0.3, 0.3, n)))
        Delta = 2.0 * rng.uniform(0, 3)
        insts.append(dict(calib=calib, Om=np.full(n, 2.0), delta=np.full(n, -Delta), edges=edges))
        codes = ref.independent_states(n, edges, None)
        pairs = [(p["i"], p["j"], p["V"]) for p in calib["pairs"]]
        w = np.linalg.eigvalsh(ref.dense_h(n, codes, np.full(n, 2.0), np.full(n, -Delta), pairs))
        want.append((w[0], w[1] - w[0]))
    want = np.array(want)
    r64 = batched_ground_states(insts, dtype="float64", tol=1e-10)
    assert r64["converged"].all()
    assert np.max(np.abs(r64["E0"] - want[:, 0])) < 1e-8
    assert np.max(np.abs(r64["gap"] - want[:, 1])) < 1e-7
    r32 = batched_ground_states(insts, dtype="float32", tune=True)
    assert np.max(np.abs(r32["E0"] - want[:, 0]) / np.abs(want[:, 0])) < 1e-6


def test_batched_graph_replay_is_deterministic(ctx):
    from energy_level_b200.batched import BatchedGroundStates
    insts = [c for c in configs.batch512(count=32)]
    b = BatchedGroundStates(insts, dtype="float32")
    b.run()
    r1 = b.results()
    g = b.capture()
    g.replay()
    r2 = b.results()
    assert np.array_equal(r1["E0"], r2["E0"])
    b.close()
