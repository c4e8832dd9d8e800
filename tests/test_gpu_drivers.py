"""GPU parity of the Krylov, KPM and Chebyshev drivers against the oracle."""
import numpy as np
import pytest

from oracle import ref
from energy_level_b200 import configs

pytestmark = pytest.mark.gpu


def _chain_model(n, seed=3):
    rng = np.random.default_rng(seed)
    om = rng.uniform(0.5, 2.0, n)
    de = rng.uniform(-2, 2, n)
    pairs = configs.pairs_from_positions(configs.chain_positions(n, jitter=rng.uniform(-0.4, 0.4, n)))
    return om, de, pairs


@pytest.mark.parametrize("kind", ["full", "chain", "ring"])
@pytest.mark.parametrize("dtype,tol", [("float64", 1e-9), ("float32", 2e-5), ("complex128", 1e-9)])
def test_lanczos_ground_matches_dense(ctx, kind, dtype, tol):
    from energy_level_b200.core import Basis, Hamiltonian
    from energy_level_b200 import solvers
    n = 10
    om, de, pairs = _chain_model(n)
    edges = {"full": None, "chain": configs.chain_edges(n), "ring": configs.ring_edges(n)}[kind]
    b = Basis(ctx, n, kind="full" if kind == "full" else "blockade", edges=edges)
    h = Hamiltonian(ctx, b, om, de, pairs)
    codes = None if kind == "full" else ref.independent_states(n, edges, None)
    w = np.linalg.eigvalsh(ref.dense_h(n, codes, om, de, pairs))
    r = solvers.lanczos_ground(h, dtype=dtype, tol=tol, nev=2)
    assert r["converged"]
    scale = max(1.0, abs(w[0]))
    etol = 1e-9 if dtype != "float32" else 1e-6
    assert abs(r["evals"][0] - w[0]) <= etol * scale
    assert abs(r["evals"][1] - w[1]) <= 10 * etol * scale


def test_chain12_ground_energy(ctx):
    """Workload chain12 (open chain N=12, full basis, FP64, tol 1e-12)."""
    from energy_level_b200.core import Basis, Hamiltonian
    from energy_level_b200 import solvers
    cfg = configs.chain12()
    b = Basis(ctx, cfg["n"], kind="full")
    pairs = [(p["i"], p["j"], p["V"]) for p in cfg["calib"]["pairs"]]
    h = Hamiltonian(ctx, b, cfg["Om"], cfg["delta"], pairs)
    r = solvers.lanczos_ground(h, dtype="float64", tol=1e-12, nev=2, max_iter=400)
    assert r["converged"]
    # reference eigsh / dense eigh value (energies in cyclic MHz)
    assert abs(r["evals"][0] - (-10.2963231346414)) < 1e-9
    assert abs((r["evals"][1] - r["evals"][0]) - 0.840389) < 1e-5


@pytest.mark.parametrize("mode", ["direct", "doubling"])
@pytest.mark.parametrize("dtype,tol", [("float64", 1e-10), ("float32", 2e-4)])
def test_kpm_moments_match_oracle(ctx, mode, dtype, tol):
    from energy_level_b200.core import Basis, Hamiltonian
    from energy_level_b200 import solvers
    n = 8
    om, de, pairs = _chain_model(n, 5)
    b = Basis(ctx, n, kind="full")
    h = Hamiltonian(ctx, b, om, de, pairs)
    H = ref.dense_h(n, None, om, de, pairs)
    emin, emax, c, r = ref.kpm_bounds(H)
    rng = np.random.default_rng(3)
    nvec, num = 6, 64
    z = rng.choice(np.array([-1.0, 1.0]), size=(nvec, 1 << n))
    want = ref.kpm_moments(lambda v: H @ v, 1 << n, num, z, c, r)
    got = solvers.kpm_moments(h, num, nvec, c, r, dtype=dtype, chunk=4, probes=z, mode=mode)
    assert np.abs(got - want).max() < tol


def test_bounds_match_dense(ctx):
    from energy_level_b200.core import Basis, Hamiltonian
    from energy_level_b200 import solvers
    n = 10
    om, de, pairs = _chain_model(n, 6)
    b = Basis(ctx, n, kind="full")
    h = Hamiltonian(ctx, b, om, de, pairs)
    w = np.linalg.eigvalsh(ref.dense_h(n, None, om, de, pairs))
    lo, hi = solvers.bounds(h, max_iter=400, tol=1e-13)
    assert abs(lo - w[0]) < 1e-8 and abs(hi - w[-1]) < 1e-8


@pytest.mark.parametrize("dtype,tol", [("complex128", 1e-9), ("complex64", 2e-5)])
def test_cheb_evolution_matches_expm(ctx, dtype, tol):
    import torch
    from energy_level_b200.core import Basis, Hamiltonian
    from energy_level_b200 import solvers
    n = 10
    edges = configs.chain_edges(n)
    om, de, pairs = _chain_model(n, 7)
    codes = ref.independent_states(n, edges, None)
    b = Basis(ctx, n, kind="blockade", edges=edges)
    h = Hamiltonian(ctx, b, om, de, pairs)
    rng = np.random.default_rng(2)
    psi0 = rng.normal(size=len(codes)) + 1j * rng.normal(size=len(codes))
    psi0 /= np.linalg.norm(psi0)
    import scipy.linalg as sla
    H = ref.dense_h(n, codes, om, de, pairs)
    want = sla.expm(-1j * ref.CONV * 37.0 * H) @ psi0
    psi = torch.as_tensor(psi0, dtype=getattr(torch, dtype), device=ctx.device)
    solvers.cheb_step(h, psi, 37.0, tol=1e-13 if dtype == "complex128" else 1e-7)
    got = psi.cpu().numpy()
    assert np.abs(got - want).max() < tol
    ns, nrm = solvers.observables(h, psi)
    assert abs(nrm - 1.0) < 10 * tol
    assert np.allclose(ns, ref.site_occupations(n, codes, want), atol=10 * tol)


@pytest.mark.parametrize("n", [8, 13, 14, 17])
@pytest.mark.parametrize("dtype,tol", [("float64", 1e-10), ("float32", 2e-4)])
def test_tiled_kpm_matches_oracle(ctx, n, dtype, tol):
    """Tiled full-basis KPM (doubling) vs the C oracle's direct recurrence on
    identical probes; n >= 14 exercises the two-group pass alternation."""
    from energy_level_b200.core import Basis, Hamiltonian
    from energy_level_b200 import solvers
    from oracle import build as ob
    rng = np.random.default_rng(n)
    om = rng.uniform(0.5, 2.0, n)
    de = rng.uniform(-3, 3, n)
    pos = [[6.0 * (i % 5), 6.0 * (i // 5), 0.0] for i in range(n)]
    pairs = configs.pairs_from_positions(pos)
    b = Basis(ctx, n, kind="full")
    h = Hamiltonian(ctx, b, om, de, pairs)
    lo, hi = solvers.bounds(h, max_iter=400, tol=1e-13)
    c, r = solvers.kpm_scale(lo, hi)
    nvec, num = 8, 41
    z = rng.choice(np.array([-1, 1], dtype=np.int8), size=(nvec, 1 << n))
    want = ob.kpm_full(n, om, ob.diag_full(n, de, pairs), c, r, num, z)
    got = solvers.kpm_moments(h, num, nvec, c, r, dtype=dtype, chunk=8, probes=z, mode="doubling")
    gen = solvers.kpm_moments(h, num, nvec, c, r, dtype=dtype, chunk=8, probes=z, mode="doubling",
                              generic=True)
    assert np.abs(got - want).max() < tol
    assert np.abs(gen - want).max() < tol


@pytest.mark.parametrize("n", [20, 21, 22, 23, 24, 25])
@pytest.mark.parametrize("dtype,tol", [("float64", 1e-10), ("float32", 2e-4)])
def test_tma_kpm_matches_generic_kernel(ctx, n, dtype, tol):
    """TMA-fed tiled KPM (20 <= N <= 25) vs the row-parallel kernel on the same
    probes, and the FP64 result vs the C oracle's direct recurrence."""
    from energy_level_b200.core import Basis, Hamiltonian
    from energy_level_b200 import solvers
    rng = np.random.default_rng(n)
    om = rng.uniform(0.5, 2.0, n)
    de = rng.uniform(-3, 3, n)
    pos = [[6.0 * (i % 5), 6.0 * (i // 5), 0.0] for i in range(n)]
    pairs = configs.pairs_from_positions(pos)
    b = Basis(ctx, n, kind="full")
    h = Hamiltonian(ctx, b, om, de, pairs)
    lo, hi = solvers.bounds(h, max_iter=400, tol=1e-12)
    c, r = solvers.kpm_scale(lo, hi)
    nvec, num = 8, 21
    z = rng.choice(np.array([-1, 1], dtype=np.int8), size=(nvec, 1 << n))
    got = solvers.kpm_moments(h, num, nvec, c, r, dtype=dtype, chunk=8, probes=z, mode="doubling")
    gen = solvers.kpm_moments(h, num, nvec, c, r, dtype="float64", chunk=8, probes=z, mode="direct",
                              generic=True)
    assert np.abs(got - gen).max() < tol
    if n == 20 and dtype == "float64":
        from oracle import build as ob
        want = ob.kpm_full(n, om, ob.diag_full(n, de, pairs), c, r, num, z[:2])
        got2 = solvers.kpm_moments(h, num, 2, c, r, dtype="float64", chunk=2, probes=z[:2])
        assert np.abs(got2 - want).max() < 1e-10


def headline_probe_block(n, distinct=4, block=32, seed=2):
    """The benchmark's probe block with the C oracle's probes in it: `distinct`
    counter-based probes, repeated to fill a block of `block` with the sign
    flipped on every second repetition.  A moment is quadratic in its probe,
    so the block mean equals the mean over the distinct probes, while each
    probe group of the pass holds data of its own (a mix-up of groups changes
    the result)."""
    from energy_level_b200.probes import rademacher_host
    z = rademacher_host(seed=seed, probe0=0, nvec=distinct, dim=1 << n)
    reps = block // distinct
    zz = np.empty((block, 1 << n), dtype=np.int8)
    for k in range(reps):
        zz[k * distinct:(k + 1) * distinct] = z if k % 2 == 0 else -z
    return z, zz


@pytest.mark.parametrize("dtype,tol", [("float64", 1e-10), ("float32", 2e-4)])
def test_tma_kpm_benchmark_shape_matches_oracle(ctx, dtype, tol):
    """The benchmark's exact shape -- 5x5 lattice (N = 25, full 2^25 basis),
    one block of 32 probes (chunk 32), doubling recurrence, TMA pass kernel --
    against the C oracle's direct recurrence (kpm.py:26-75 / 115-151) on the
    same probes, 24 moments."""
    from energy_level_b200.core import Basis, Hamiltonian
    from energy_level_b200 import solvers
    from oracle import build as ob
    cfg = configs.square25()
    n = cfg["n"]
    pairs = [(p["i"], p["j"], p["V"]) for p in cfg["calib"]["pairs"]]
    d = ob.diag_full(n, cfg["delta"], pairs)
    half = 0.5 * float(np.sum(np.abs(cfg["Om"])))
    lo, hi = float(d.min()) - half, float(d.max()) + half   # a rigorous spectral interval
    c, r = solvers.kpm_scale(lo, hi)
    num = 24
    z, zz = headline_probe_block(n)
    want = ob.kpm_full(n, cfg["Om"], d, c, r, num, z)
    b = Basis(ctx, n, kind="full")
    h = Hamiltonian(ctx, b, cfg["Om"], cfg["delta"], pairs)
    got = solvers.kpm_moments(h, num, 32, c, r, dtype=dtype, chunk=32, probes=zz, mode="doubling")
    assert abs(got[0] - 1.0) < 1e-12
    assert np.abs(got - want).max() < tol


def _oracle_extremes(n, om, d, steps=300, seed=0):
    """Extremal eigenvalues by a plain Lanczos run on the C oracle's H x."""
    import ctypes as C
    from scipy.linalg import eigvalsh_tridiagonal
    from oracle import build as ob
    lib = ob.load()
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    om = np.ascontiguousarray(om, dtype=np.float64)
    d = np.ascontiguousarray(d, dtype=np.float64)

    def hv(x):
        y = np.empty_like(x)
        lib.oracle_apply_full(n, dp(om), dp(d), 1, 1.0, 0.0, 0.0, dp(x), None, dp(y))
        return y
    v = np.random.default_rng(seed).standard_normal(1 << n)
    v /= np.linalg.norm(v)
    vp = np.zeros_like(v)
    al, be, beta = [], [], 0.0
    for _ in range(steps):
        w = hv(v) - beta * vp
        a = float(v @ w)
        w -= a * v
        al.append(a)
        beta = float(np.linalg.norm(w))
        be.append(beta)
        vp, v = v, w / beta
    ev = eigvalsh_tridiagonal(np.array(al), np.array(be[:-1]))
    return ev[0], ev[-1]


@pytest.mark.parametrize("n", [20, 21])
def test_tiled_bounds_match_oracle_lanczos(ctx, n):
    """Spectral bounds of the full basis at N >= 20, where the FP64 Lanczos
    runs the tiled two-pass product (A tiles, then B pieces), against a
    Lanczos run on the C oracle's H x (the reference's kpm._bounds role,
    kpm.py:82-97)."""
    from energy_level_b200.core import Basis, Hamiltonian
    from energy_level_b200 import solvers
    from oracle import build as ob
    rng = np.random.default_rng(40 + n)
    om = rng.uniform(0.5, 2.0, n)
    de = rng.uniform(-3, 3, n)
    pos = [[6.0 * (i % 5), 6.0 * (i // 5), 0.0] for i in range(n)]
    pairs = configs.pairs_from_positions(pos)
    lo_want, hi_want = _oracle_extremes(n, om, ob.diag_full(n, de, pairs))
    h = Hamiltonian(ctx, Basis(ctx, n, kind="full"), om, de, pairs)
    lo, hi = solvers.bounds(h, max_iter=400, tol=1e-12)
    scale = max(abs(lo_want), abs(hi_want))
    assert abs(lo - lo_want) < 1e-9 * scale and abs(hi - hi_want) < 1e-9 * scale
