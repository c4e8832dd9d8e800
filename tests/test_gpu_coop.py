"""GPU parity of the cooperative single-instance Lanczos (el_batch_run_coop):
every instance solved by one cooperative launch over up to 64 CTAs, against
dense eigenvalues from the oracle and the reference's C1 ground energy."""
import numpy as np
import pytest

from oracle import ref
from energy_level_b200 import configs

pytestmark = pytest.mark.gpu

C1_E0 = -10.2963231346414      # 12-site chain, full basis (the reference's ground_state)


def _dense(n, edges, om, de, calib):
    codes = None if edges is None else ref.independent_states(n, edges, None)
    pairs = [(p["i"], p["j"], p["V"]) for p in calib["pairs"]]
    w = np.linalg.eigvalsh(ref.dense_h(n, codes, om, de, pairs))
    return w[0], w[1] - w[0]


@pytest.mark.parametrize("dtype,tol_e", [("float64", 1e-9), ("float32", 2e-6)])
def test_coop_c1_matches_reference(ctx, dtype, tol_e):
    from energy_level_b200.batched import BatchedGroundStates
    cfg = configs.chain12()
    inst = [dict(calib=cfg["calib"], Om=cfg["Om"], delta=cfg["delta"], edges=None)]
    b = BatchedGroundStates(inst, dtype=dtype, max_iter=300, tol=1e-10 if dtype == "float64" else 1e-5)
    b.run_coop()
    r = b.results()
    e0, gap = _dense(12, None, cfg["Om"], cfg["delta"], cfg["calib"])
    assert abs(e0 - C1_E0) < 1e-9
    assert r["converged"][0]
    assert abs(r["E0"][0] - e0) < tol_e * max(1.0, abs(e0))
    assert abs(r["gap"][0] - gap) < (1e-7 if dtype == "float64" else 1e-4)
    # a second run gives the same bits (fixed-order reductions)
    b.run_coop()
    assert b.results()["E0"][0] == r["E0"][0]
    b.close()


def test_coop_several_instances_match_dense(ctx):
    from energy_level_b200.batched import BatchedGroundStates
    rng = np.random.default_rng(6)
    insts, want = [], []
    for k, (n, kind) in enumerate([(14, "chain"), (13, "ring"), (10, "full"), (16, "chain"), (9, "ring")]):
        edges = None if kind == "full" else (configs.ring_edges(n) if kind == "ring" else configs.chain_edges(n))
        calib = configs.calib_from_positions(configs.chain_positions(n, jitter=rng.uniform(-0.3, 0.3, n)))
        om, de = np.full(n, 2.0), np.full(n, -2.0 * rng.uniform(0, 3))
        insts.append(dict(calib=calib, Om=om, delta=de, edges=edges))
        want.append(_dense(n, edges, om, de, calib))
    want = np.array(want)
    b = BatchedGroundStates(insts, dtype="float64", max_iter=300, tol=1e-10)
    b.run_coop()
    r = b.results()
    assert r["converged"].all()
    assert np.max(np.abs(r["E0"] - want[:, 0])) < 1e-8
    assert np.max(np.abs(r["gap"] - want[:, 1])) < 1e-7
    # the single-CTA persistent kernel agrees
    b.run()
    r2 = b.results()
    assert np.max(np.abs(r2["E0"] - r["E0"])) < 1e-8
    b.close()


def test_coop_refuses_too_large_instance(ctx):
    from energy_level_b200.batched import BatchedGroundStates
    n = 28                          # chain sector of 832,040 rows: more than 64 x 1024
    calib = configs.calib_from_positions(configs.chain_positions(n))
    b = BatchedGroundStates([dict(calib=calib, Om=np.full(n, 2.0), delta=np.zeros(n),
                                  edges=configs.chain_edges(n))], dtype="float32", max_iter=50)
    with pytest.raises(ValueError):
        b.run_coop()
    b.close()


def test_coop_check_interval_and_passes_agree(ctx):
    """The same C1 ground energy for other check intervals and one pass."""
    from energy_level_b200.batched import BatchedGroundStates
    cfg = configs.chain12()
    inst = [dict(calib=cfg["calib"], Om=cfg["Om"], delta=cfg["delta"], edges=None)]
    b = BatchedGroundStates(inst, dtype="float64", max_iter=300, tol=1e-10)
    for ce, ps in ((8, 2), (16, 2), (8, 1)):
        b.run_coop(check_every=ce, reorth_passes=ps)
        r = b.results()
        assert r["converged"][0] and abs(r["E0"][0] - C1_E0) < 1e-9, (ce, ps)
    b.close()


def test_coop_barrier_timeout_is_reported_and_the_context_recovers(ctx):
    """A grid-barrier wait bounded at zero polls runs out in the first of two
    instances: el_batch_run_coop returns EL_ECUDA (RuntimeError, 'grid
    barrier timed out') instead of hanging or returning stale energies, and
    with the default bound restored the same batch solves normally on the
    same context.  No asynchronous copy is in flight in this kernel, so a
    CTA that stops waiting leaves nothing behind."""
    from energy_level_b200.batched import BatchedGroundStates
    cfg = configs.chain12()
    n = 10
    calib = configs.calib_from_positions(configs.chain_positions(n))
    inst = [dict(calib=cfg["calib"], Om=cfg["Om"], delta=cfg["delta"], edges=None),
            dict(calib=calib, Om=np.full(n, 2.0), delta=np.full(n, -1.0), edges=None)]
    b = BatchedGroundStates(inst, dtype="float64", max_iter=300, tol=1e-10)
    b.set_wait_limit(0)
    with pytest.raises(RuntimeError, match="grid barrier timed out"):
        b.run_coop()
    b.set_wait_limit()
    b.run_coop()
    r = b.results()
    assert r["converged"].all()
    assert abs(r["E0"][0] - C1_E0) < 1e-9
    with pytest.raises(ValueError):
        b.set_wait_limit(-1)
    b.close()


@pytest.mark.parametrize("mode", ["batch", "coop"])
def test_batched_occupations_match_dense_ground_states(ctx, mode):
    """n_atom of the batched solvers (persistent and cooperative) against the
    occupations of the dense ground-state eigenvectors, as the reference's
    batched_ground_state returns them (equilibrium.py:251-311)."""
    from energy_level_b200.batched import batched_ground_states
    rng = np.random.default_rng(12)
    insts, want = [], []
    for n, kind in [(12, "full"), (14, "chain"), (11, "ring"), (16, "chain")]:
        edges = None if kind == "full" else (configs.ring_edges(n) if kind == "ring" else configs.chain_edges(n))
        calib = configs.calib_from_positions(configs.chain_positions(n, jitter=rng.uniform(-0.3, 0.3, n)))
        om, de = np.full(n, 2.0), rng.uniform(-3.0, 1.0, n)
        insts.append(dict(calib=calib, Om=om, delta=de, edges=edges))
        codes = None if edges is None else ref.independent_states(n, edges, None)
        pairs = [(p["i"], p["j"], p["V"]) for p in calib["pairs"]]
        w, v = np.linalg.eigh(ref.dense_h(n, codes, om, de, pairs))
        want.append(ref.site_occupations(n, codes, v[:, 0]))
    out = batched_ground_states(insts, dtype="float64", max_iter=300, tol=1e-11, mode=mode)
    assert out["mode"] == mode and out["converged"].all()
    for i, inst in enumerate(insts):
        n = len(inst["Om"])
        assert np.max(np.abs(out["n_atom"][i, :n] - want[i])) < 1e-7, i
        assert np.all(out["n_atom"][i, n:] == 0)
