"""Pin the CPU oracle to golden vectors written by the reference itself
(tests/golden/make_golden.py).  CPU only."""
import os

import numpy as np
import pytest

from oracle import ref

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLD, name + ".npz"), allow_pickle=False)


def pairs_of(arr):
    return [(int(i), int(j), float(v)) for i, j, v in np.asarray(arr)]


@pytest.mark.parametrize("name", ["chain10", "ring11", "ring20", "square3x3", "nnn_chain12", "chain22"])
def test_independent_states_bit_exact(name):
    g = load("basis")
    n = int(g["n_" + name])
    edges = g["edges_" + name].tolist()
    codes = ref.independent_states(n, edges, max_states=None)
    assert np.array_equal(codes, g["codes_" + name])
    assert len(codes) == int(g["count_" + name])


def test_fibonacci_and_lucas_dimensions():
    g = load("basis")
    assert len(g["codes_chain22"]) == ref.fib(24)
    assert len(g["codes_ring20"]) == ref.fib(21) + ref.fib(19) == 15127
    assert len(g["codes_chain10"]) == ref.fib(12)


@pytest.mark.parametrize("n,k", [(10, 4), (12, 6), (6, 0), (6, 6)])
def test_number_sector_bit_exact(n, k):
    g = load("basis")
    assert np.array_equal(ref.number_sector_basis(n, k), g["charge_%d_%d" % (n, k)])


def test_max_states_cap():
    with pytest.raises(ValueError):
        ref.independent_states(20, [[i, i + 1] for i in range(19)], max_states=100)


@pytest.mark.parametrize("name", ["full7", "chain10", "ring9", "square3x3", "cplx8"])
def test_hv_matches_reference(name):
    g = load("hv")
    n = int(g["n_" + name])
    edges = g["edges_" + name].tolist()
    codes = None if not edges else ref.independent_states(n, edges, None)
    y = ref.hv(n, codes, g["om_" + name], g["de_" + name], pairs_of(g["pairs_" + name]), g["x_" + name])
    assert np.max(np.abs(y - g["y_" + name])) < 1e-12 * max(1.0, np.abs(g["y_" + name]).max())


@pytest.mark.parametrize("name", ["full7", "chain10", "ring9", "square3x3"])
def test_diagonal_matches_reference(name):
    g = load("hv")
    n = int(g["n_" + name])
    edges = g["edges_" + name].tolist()
    codes = np.arange(1 << n) if not edges else ref.independent_states(n, edges, None)
    d = ref.diagonal(n, codes, g["de_" + name], pairs_of(g["pairs_" + name]))
    assert np.max(np.abs(d - g["diag_" + name])) < 1e-12


def test_kpm_matches_reference():
    g = load("kpm")
    n = int(g["n"])
    H = ref.dense_h(n, None, g["om"], g["de"], pairs_of(g["pairs"]))
    emin, emax, c, r = ref.kpm_bounds(H)
    assert abs(emin - float(g["emin"])) < 1e-9 and abs(emax - float(g["emax"])) < 1e-9
    assert abs(c - float(g["c"])) < 1e-9 and abs(r - float(g["r"])) < 1e-9
    num = int(g["num"])
    mu = ref.kpm_moments(lambda v: H @ v, H.shape[0], num, g["probes"], float(g["c"]), float(g["r"]))
    assert np.max(np.abs(mu - g["mu"])) < 1e-12
    mu_ex = ref.kpm_moments_exact(H, num, float(g["c"]), float(g["r"]))
    assert np.max(np.abs(mu_ex - g["mu_exact"])) < 1e-12
    assert np.max(np.abs(ref.jackson_kernel(num) - g["jackson"])) < 1e-15
    rho = ref.dos_from_moments(g["mu"], float(g["c"]), float(g["r"]), g["energies"], num)
    assert np.max(np.abs(rho - g["rho"])) < 1e-12


def test_kpm_doubling_identity_matches_direct():
    """mu_2n = 2<T_n z, T_n z> - mu_0 and mu_2n+1 = 2<T_n+1 z, T_n z> - mu_1
    reproduce the direct recurrence (the identity the GPU doubling mode uses)."""
    g = load("kpm")
    n = int(g["n"])
    H = ref.dense_h(n, None, g["om"], g["de"], pairs_of(g["pairs"]))
    c, r = float(g["c"]), float(g["r"])
    Ht = (H - c * np.eye(H.shape[0])) / r
    num = int(g["num"])
    acc = np.zeros(num + 1)
    for z in g["probes"]:
        ts = [z, Ht @ z]
        while len(ts) < num // 2 + 2:
            ts.append(2 * Ht @ ts[-1] - ts[-2])
        m0, m1 = z @ z, ts[1] @ z
        acc[0] += m0
        acc[1] += m1
        for k in range(1, num // 2 + 1):
            if 2 * k <= num:
                acc[2 * k] += 2 * ts[k] @ ts[k] - m0
            if 2 * k + 1 <= num:
                acc[2 * k + 1] += 2 * ts[k + 1] @ ts[k] - m1
    mu = acc / (len(g["probes"]) * H.shape[0])
    assert np.max(np.abs(mu - g["mu"])) < 1e-11


def test_ground_state_chain12_matches_reference():
    g = load("ground")
    from energy_level_b200 import configs
    cfg = configs.chain12()
    pairs = [(p["i"], p["j"], p["V"]) for p in cfg["calib"]["pairs"]]
    codes = ref.independent_states(12, configs.chain_edges(12), None)
    w = np.linalg.eigvalsh(ref.dense_h(12, codes, cfg["Om"], cfg["delta"], pairs))
    assert abs(w[0] - float(g["chain12b_E0"])) < 1e-9
    assert abs((w[1] - w[0]) - float(g["chain12b_gap"])) < 1e-9
    # full basis value quoted by the reference (eigsh on the matrix-free operator)
    assert abs(float(g["chain12_E0"]) - (-10.2963231346414)) < 1e-9


def test_evolution_matches_reference():
    g = load("evolve")
    n = int(g["n"])
    from energy_level_b200 import configs
    segs = [{"t0": float(t), "Om": om, "delta": de} for t, om, de in zip(g["seg_t0"], g["seg_om"], g["seg_de"])]
    codes = ref.independent_states(n, configs.chain_edges(n), None)
    assert np.array_equal(codes, g["basis_states"])
    psi0 = np.zeros(len(codes), complex)
    psi0[0] = 1.0
    states = ref.evolve_segments(n, codes, pairs_of(g["pairs"]), segs, psi0, g["t_grid"])
    assert np.max(np.abs(states[-1] - g["psi_final"])) < 1e-10
    pops = np.array([ref.site_occupations(n, codes, s) for s in states])
    assert np.max(np.abs(pops - g["pops_atom"])) < 1e-10


def exchange_case(g, name):
    """(n, codes, om, de, V pairs, exchange) of one exchange fixture case."""
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
    codes = g["codes_" + name]
    full = len(codes) == (1 << n)
    return n, (None if full else codes), g["om_" + name], g["de_" + name], pairs, ex


@pytest.mark.parametrize("name", ["full7", "charge10_4", "charge9_3c", "chain10"])
def test_exchange_hv_matches_reference(name):
    g = load("exchange")
    n, codes, om, de, pairs, ex = exchange_case(g, name)
    y = ref.hv(n, codes, om, de, pairs, g["x_" + name], exchange=ex)
    assert np.max(np.abs(y - g["y_" + name])) < 1e-12 * max(1.0, np.abs(g["y_" + name]).max())


def test_exchange_hermitian_and_sparse_agree():
    g = load("exchange")
    n, codes, om, de, pairs, ex = exchange_case(g, "full7")
    H = ref.dense_h(n, codes, om, de, pairs, exchange=ex)
    assert np.allclose(H, H.conj().T, atol=1e-14)
    S = ref.sparse_h(n, codes, om, de, pairs, exchange=ex).toarray()
    assert np.max(np.abs(S - H)) < 1e-14


def test_sector_scan_matches_reference():
    from energy_level_b200 import configs
    g = load("exchange")
    xy = configs.xy_chain(10)
    pairs = [(p['i'], p['j'], p['V']) for p in xy['calib']['pairs']]
    ex = [(p['i'], p['j'], p['J'], 0.0) for p in xy['calib']['pairs']]
    E0, k, rows = ref.sector_scan(10, xy['delta'], pairs, ex)
    assert k == int(g["scan_sector"])
    assert abs(E0 - float(g["scan_E0"])) < 1e-10
    assert np.allclose([r[2] for r in rows], g["scan_sector_E0"], atol=1e-10, rtol=0)
    assert np.array_equal([r[1] for r in rows], g["scan_sector_dim"])
    assert sum(r[1] for r in rows) == int(g["scan_dimension_sum"]) == 1 << 10
    # the lowest sector energy is the full-basis ground energy
    Hf = ref.dense_h(10, None, np.zeros(10), xy['delta'], pairs, exchange=ex)
    assert abs(np.linalg.eigvalsh(Hf)[0] - E0) < 1e-10


def test_sector_ground_corr_matches_reference():
    from energy_level_b200 import configs
    g = load("exchange")
    xy = configs.xy_chain(10)
    pairs = [(p['i'], p['j'], p['V']) for p in xy['calib']['pairs']]
    ex = [(p['i'], p['j'], p['J'], 0.0) for p in xy['calib']['pairs']]
    codes = ref.number_sector_basis(10, 5)
    assert np.array_equal(codes, g["gs5_sector_idx"])
    w, V = np.linalg.eigh(ref.dense_h(10, codes, np.zeros(10), xy['delta'], pairs, exchange=ex))
    assert abs(w[0] - float(g["gs5_E0"])) < 1e-10
    p = np.abs(V[:, 0]) ** 2
    bits = ref.basis_bits(10, codes)
    assert np.allclose(bits @ p, g["gs5_n_atom"], atol=1e-9)
    assert np.allclose(ref.corr_matrix(bits, p), g["gs5_corr"], atol=1e-9)


@pytest.mark.parametrize("which", ["full", "basis"])
def test_spin_observables_match_reference(which):
    g = load("observables")
    if which == "full":
        n, codes, psi = 7, None, g["full_psi"]
    else:
        n, codes, psi = 10, g["basis_states"], g["basis_psi"]
    ob = ref.spin_observables(n, codes, psi)
    for k in ("sx", "sy", "sz", "sp", "sm", "xy_corr"):
        assert np.allclose(ob[k], g["%s_%s" % (which, k)], atol=1e-12, rtol=0), k
    assert np.allclose(ob["phase"], g[which + "_phase"], atol=1e-12, rtol=0, equal_nan=True)


def test_entropies_and_corr_match_reference():
    g = load("observables")
    assert abs(ref.entropy_cut(7, None, g["full_psi"], 3) - float(g["full_S3"])) < 1e-12
    assert abs(ref.entropy_cut(10, g["basis_states"], g["basis_psi"], 5) - float(g["basis_S5"])) < 1e-12
    bits = ref.basis_bits(10, g["basis_states"])
    assert np.allclose(ref.corr_matrix(bits, np.abs(g["basis_psi"]) ** 2), g["basis_corr"], atol=1e-13)


@pytest.mark.parametrize("name", ["full7", "chain10"])
def test_loss_hv_matches_reference(name):
    from energy_level_b200 import configs
    g = load("loss")
    n = 7 if name == "full7" else 10
    calib = configs.calib_from_positions(configs.chain_positions(n))
    pairs = [(p["i"], p["j"], p["V"]) for p in calib["pairs"]]
    codes = None if name == "full7" else ref.independent_states(n, configs.chain_edges(n), None)
    p = "hv_" + name + "_"
    y = ref.hv(n, codes, g[p + "om"], g[p + "de"], pairs, g[p + "x"], gamma=g[p + "ga"])
    assert np.max(np.abs(y - g[p + "y"])) < 1e-12 * max(1.0, np.abs(g[p + "y"]).max())


def test_loss_evolution_oracle_matches_reference():
    from energy_level_b200 import configs
    g = load("loss")
    n = 6
    xy = configs.xy_chain(n, seed=31)
    pairs = [(p["i"], p["j"], p["V"]) for p in xy["calib"]["pairs"]]
    ex = [(p["i"], p["j"], p["J"], 0.0) for p in xy["calib"]["pairs"]]
    segs = [{"t0": float(t0), "Om": om, "delta": de}
            for t0, om, de in zip(g["ev1_seg_t0"], g["ev1_seg_om"], g["ev1_seg_de"])]
    psi0 = np.zeros(1 << n, complex)
    psi0[int("10" * 3, 2)] = 1.0
    out = ref.evolve_segments(n, None, pairs, segs, psi0, g["ev1_t"], exchange=ex, gamma=g["ev1_ga"])
    norms = np.asarray([np.vdot(v, v).real for v in out])
    assert np.allclose(norms, g["ev1_norms"], atol=1e-10, rtol=0)
    assert np.abs(out[-1] - g["ev1_psi_amp"]).max() < 1e-10
