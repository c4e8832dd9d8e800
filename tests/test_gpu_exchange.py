"""GPU parity of the exchange channels (I2 J, I3 A) and the sector scan
against golden vectors written by the reference and against the oracle."""
import os

import numpy as np
import pytest

from oracle import ref
from energy_level_b200 import configs

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["full7", "charge10_4", "charge9_3c", "chain10"]


def gold():
    return np.load(os.path.join(GOLD, "exchange.npz"))


def case(g, name):
    n = int(g["n_" + name])
    terms = set(str(t) for t in g["terms_" + name])
    ij = g["pairs_" + name]
    pairs = [(int(i), int(j), float(v)) for (i, j), v in zip(ij, g["V_" + name])] if "I1" in terms else []
    ex = []
    for (i, j), J, A in zip(ij, g["J_" + name], g["A_" + name]):
        J = complex(J) if "I2" in terms else 0j
        A = complex(A) if "I3" in terms else 0j
        if J != 0 or A != 0:
            ex.append((int(i), int(j), J, A))
    return n, pairs, ex


def basis_of(ctx, name, n):
    from energy_level_b200.core import Basis
    if name.startswith("full"):
        return Basis(ctx, n, kind="full")
    if name.startswith("charge"):
        k = int(name.split("_")[1].rstrip("c"))
        return Basis(ctx, n, kind="charge", k=k)
    return Basis(ctx, n, kind="blockade", edges=configs.chain_edges(n))


@pytest.mark.parametrize("name", CASES)
def test_exchange_hv_matches_reference(ctx, name):
    import torch
    from energy_level_b200.core import Hamiltonian
    g = gold()
    n, pairs, ex = case(g, name)
    b = basis_of(ctx, name, n)
    assert np.array_equal(b.codes().cpu().numpy(), g["codes_" + name])
    h = Hamiltonian(ctx, b, g["om_" + name], g["de_" + name], pairs, exchange=ex)
    x = torch.as_tensor(g["x_" + name], dtype=torch.complex128, device=ctx.device)
    want = g["y_" + name]
    got = h.hv(x).cpu().numpy()
    assert np.abs(got - want).max() <= 1e-12 * max(1.0, np.abs(want).max())
    # single precision, block of 4 vectors
    X = torch.stack([x * (1 + 0.5 * k) for k in range(4)], dim=1).to(torch.complex64).contiguous()
    got4 = h.hv(X).cpu().numpy()
    want4 = np.stack([want * (1 + 0.5 * k) for k in range(4)], axis=1)
    assert np.abs(got4 - want4).max() <= 2e-5 * max(1.0, np.abs(want4).max())


@pytest.mark.parametrize("name", ["charge10_4", "chain10"])
def test_exchange_real_hv_float64(ctx, name):
    """Real J/A and real Omega: the real vector path gives the same product."""
    import torch
    from energy_level_b200.core import Hamiltonian
    g = gold()
    n, pairs, ex = case(g, name)
    b = basis_of(ctx, name, n)
    om = g["om_" + name].real
    h = Hamiltonian(ctx, b, om, g["de_" + name], pairs, exchange=ex)
    assert not h.complex_drive
    x = g["x_" + name].real.copy()
    want = ref.hv(n, g["codes_" + name], om, g["de_" + name], pairs, x, exchange=ex)
    for dt, tol in (("float64", 1e-12), ("float32", 2e-5)):
        got = h.hv(torch.as_tensor(x, dtype=getattr(torch, dt), device=ctx.device)).cpu().numpy()
        assert np.abs(got - want).max() <= tol * max(1.0, np.abs(want).max()), dt


def test_complex_exchange_needs_complex_dtype(ctx):
    import torch
    from energy_level_b200.core import Hamiltonian
    g = gold()
    n, pairs, ex = case(g, "charge9_3c")
    b = basis_of(ctx, "charge9_3c", n)
    h = Hamiltonian(ctx, b, np.zeros(n), g["de_charge9_3c"], pairs, exchange=ex)
    assert h.complex_drive
    with pytest.raises(ValueError):
        h.hv(torch.ones(b.dim, dtype=torch.float64, device=ctx.device))
    h.set_exchange([])
    assert not h.complex_drive
    h.hv(torch.ones(b.dim, dtype=torch.float64, device=ctx.device))


def test_sector_ground_state_matches_reference(ctx):
    from energy_level_b200 import backends
    g = gold()
    xy = configs.xy_chain(10)
    r = backends.solve_equilibrium({"calib": xy["calib"], "Om": np.zeros(10), "delta": xy["delta"],
                                    "terms": ["I1", "I2"]}, want="gs", sector=5)
    assert abs(r["E0"] - float(g["gs5_E0"])) < 1e-8
    assert abs(r["gap"] - float(g["gs5_gap"])) < 1e-7
    assert np.array_equal(r["sector_idx"], g["gs5_sector_idx"])
    assert np.allclose(r["n_atom"], g["gs5_n_atom"], atol=1e-7)


def test_sector_scan_matches_reference(ctx):
    from energy_level_b200.sector_scan import scan_ground_sectors
    g = gold()
    xy = configs.xy_chain(10)
    seen = []
    r = scan_ground_sectors(xy["calib"], delta=xy["delta"], Om=np.zeros(10), terms=["I1", "I2"],
                            progress=seen.append)
    assert r["sector"] == int(g["scan_sector"])
    assert abs(r["E0"] - float(g["scan_E0"])) < 1e-8
    assert np.allclose([row["E0"] for row in r["per_sector"]], g["scan_sector_E0"], atol=1e-8, rtol=0)
    assert [row["dim"] for row in r["per_sector"]] == g["scan_sector_dim"].tolist()
    gaps = np.asarray([row["gap"] for row in r["per_sector"]])
    assert np.allclose(gaps, g["scan_sector_gap"], atol=1e-6, rtol=0)
    assert r["dimension_sum"] == int(g["scan_dimension_sum"]) == r["full_dimension"]
    assert r["converged"] and len(seen) == 11
    assert r["sectors_run"] == list(range(11))
    assert all(set(row) >= {"sector", "dim", "E0", "gap", "residual", "converged", "backend", "seconds"}
               for row in r["per_sector"])


def test_sector_scan_larger_matches_oracle(ctx):
    """N = 14 dipolar XY chain, sectors 5..9: per-sector E0 vs the oracle."""
    from energy_level_b200.sector_scan import scan_ground_sectors
    xy = configs.xy_chain(14, seed=11)
    pairs = [(p["i"], p["j"], p["V"]) for p in xy["calib"]["pairs"]]
    ex = [(p["i"], p["j"], p["J"], 0.0) for p in xy["calib"]["pairs"]]
    ks = [5, 6, 7, 8, 9]
    r = scan_ground_sectors(xy["calib"], delta=xy["delta"], Om=np.zeros(14), terms=["I1", "I2"], sectors=ks)
    E0, k, rows = ref.sector_scan(14, xy["delta"], pairs, ex, sectors=ks)
    assert r["sector"] == k
    assert np.allclose([row["E0"] for row in r["per_sector"]], [row[2] for row in rows], atol=1e-8, rtol=0)


def test_sector_scan_refusals(ctx):
    from energy_level_b200.sector_scan import scan_ground_sectors
    xy = configs.xy_chain(6)
    with pytest.raises(ValueError):
        scan_ground_sectors(xy["calib"], delta=xy["delta"], Om=np.full(6, 0.1), terms=["I1", "I2"])
    with pytest.raises(ValueError):
        scan_ground_sectors(xy["calib"], delta=xy["delta"], Om=np.zeros(6), terms=["I1", "I2"],
                            sectors=[0, 7])
    with pytest.raises(ValueError):
        scan_ground_sectors(xy["calib"], delta=xy["delta"], gamma=np.full(6, 0.1))
    cal = dict(xy["calib"])
    cal["pairs"] = [dict(p, A=0.1) for p in cal["pairs"]]
    cal["terms"] = ["I1", "I2", "I3"]
    with pytest.raises(ValueError):
        scan_ground_sectors(cal, delta=xy["delta"], Om=np.zeros(6), terms=["I1", "I2", "I3"])


def test_exchange_evolution_matches_oracle(ctx):
    """Quench of a Neel state under XY exchange plus a drive, full basis."""
    from energy_level_b200.engine import evolve_manybody
    n = 8
    xy = configs.xy_chain(n, seed=3)
    om = np.full(n, 0.3)
    pairs = [(p["i"], p["j"], p["V"]) for p in xy["calib"]["pairs"]]
    ex = [(p["i"], p["j"], p["J"], 0.0) for p in xy["calib"]["pairs"]]
    t = np.linspace(0.0, 400.0, 5)
    r = evolve_manybody(xy["calib"], "rg" * (n // 2), t, Om=om, delta=xy["delta"], terms=["I1", "I2"],
                        record_psi=True)
    psi0 = np.zeros(1 << n, complex)
    psi0[int("10" * (n // 2), 2)] = 1.0
    seg = [{"t0": 0.0, "Om": om, "delta": xy["delta"]}]
    want = ref.evolve_segments(n, None, pairs, seg, psi0, t, exchange=ex)
    assert np.abs(r["psi_amp"] - want[-1]).max() < 1e-8
    occ = np.asarray([ref.site_occupations(n, None, w) for w in want])
    assert np.allclose(r["pops_atom"], occ, atol=1e-8)


def test_exchange_lanczos_full_basis_matches_oracle(ctx):
    """Ground state with complex J and A and a complex drive on the full basis."""
    from energy_level_b200.matrix_free import b200_lanczos_ground_state
    g = gold()
    n, pairs, ex = case(g, "full7")
    calib = {"atoms": [{"id": i, "pos": [float(i), 0, 0]} for i in range(n)],
             "pairs": [{"i": i, "j": j, "V": v, "J": 0.0, "A": 0.0} for i, j, v in pairs],
             "terms": ["I1", "I2", "I3"]}
    jmap = {(i, j): (J, A) for i, j, J, A in ex}
    for p in calib["pairs"]:
        p["J"], p["A"] = jmap.get((p["i"], p["j"]), (0j, 0j))
    r = b200_lanczos_ground_state(calib, g["om_full7"], g["de_full7"], terms=["I1", "I2", "I3"],
                                  dtype="complex128", tol=1e-11)
    w = np.linalg.eigvalsh(ref.dense_h(n, None, g["om_full7"], g["de_full7"], pairs, exchange=ex))
    assert r["converged"]
    assert abs(r["E0"] - w[0]) < 1e-9
    assert abs(r["gap"] - (w[1] - w[0])) < 1e-8


def test_exchange_kpm_generic_matches_oracle(ctx):
    """KPM moments of an XY chain (full basis, exchange -> generic recurrence)
    on explicit probes, against the oracle recurrence."""
    from energy_level_b200.kpm import kpm_moments_b200
    n = 10
    xy = configs.xy_chain(n, seed=5)
    pairs = [(p["i"], p["j"], p["V"]) for p in xy["calib"]["pairs"]]
    ex = [(p["i"], p["j"], p["J"], 0.0) for p in xy["calib"]["pairs"]]
    om = np.full(n, 0.4)
    rng = np.random.default_rng(9)
    probes = rng.choice([-1, 1], size=(4, 1 << n)).astype(np.int8)
    sys_ = {"calib": xy["calib"], "Om": om, "delta": xy["delta"], "terms": ["I1", "I2"]}
    mu, c, r = kpm_moments_b200(sys_, num=40, nvec=4, dtype="float64", probes=probes, chunk=4)
    H = ref.dense_h(n, None, om, xy["delta"], pairs, exchange=ex)
    want = ref.kpm_moments(lambda v: H @ v, 1 << n, 40, probes.astype(float), c, r)
    assert np.abs(np.asarray(mu) - want).max() < 1e-10


def test_batched_refuses_exchange(ctx):
    from energy_level_b200 import batched
    from energy_level_b200.model import ConfigConflict
    xy = configs.xy_chain(8)
    inst = {"calib": xy["calib"], "Om": np.full(8, 1.0), "delta": xy["delta"],
            "edges": configs.chain_edges(8)}
    with pytest.raises(ConfigConflict):
        batched.batched_ground_states([inst])


def test_sector_scan_workers_give_identical_rows(ctx):
    """One worker or four (separate contexts and streams): the same results."""
    from energy_level_b200.sector_scan import scan_ground_sectors
    xy = configs.xy_chain(12, seed=2)
    r1 = scan_ground_sectors(xy["calib"], delta=xy["delta"], Om=np.zeros(12), terms=["I1", "I2"], workers=1)
    r4 = scan_ground_sectors(xy["calib"], delta=xy["delta"], Om=np.zeros(12), terms=["I1", "I2"], workers=4)
    assert [r["E0"] for r in r1["per_sector"]] == [r["E0"] for r in r4["per_sector"]]
    assert [r["gap"] for r in r1["per_sector"]] == [r["gap"] for r in r4["per_sector"]]
    assert r1["sector"] == r4["sector"] and r1["converged"] and r4["converged"]
