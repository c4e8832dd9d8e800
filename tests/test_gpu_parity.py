"""GPU parity of the native kernels against the CPU oracle (through the C ABI)."""
import numpy as np
import pytest

from oracle import ref
from energy_level_b200 import configs

pytestmark = pytest.mark.gpu

GRAPHS = [
    ("chain", 10, configs.chain_edges(10), "blockade", None),
    ("ring", 11, configs.ring_edges(11), "blockade", None),
    ("square3x3", 9, [[0, 1], [1, 2], [3, 4], [4, 5], [6, 7], [7, 8], [0, 3], [3, 6], [1, 4],
                      [4, 7], [2, 5], [5, 8]], "blockade", None),
    ("nnn_chain", 12, configs.chain_edges(12) + [[i, i + 2] for i in range(10)], "blockade", None),
    ("charge", 10, None, "charge", 4),
    ("full", 8, None, "full", None),
]


def oracle_codes(n, edges, kind, k):
    if kind == "blockade":
        return ref.independent_states(n, edges, max_states=None)
    if kind == "charge":
        return ref.number_sector_basis(n, k)
    return np.arange(1 << n, dtype=np.int64)


@pytest.mark.parametrize("name,n,edges,kind,k", GRAPHS)
def test_basis_codes_and_rank_bit_exact(ctx, name, n, edges, kind, k):
    from energy_level_b200.core import Basis
    b = Basis(ctx, n, kind=kind, edges=edges, k=k)
    want = oracle_codes(n, edges, kind, k)
    got = b.codes().cpu().numpy()
    assert b.dim == len(want)
    assert np.array_equal(got, want)
    import torch
    ranks = b.rank(torch.arange(1 << n, dtype=torch.int64)).cpu().numpy()
    exp = np.full(1 << n, -1, np.int64)
    exp[want] = np.arange(len(want))
    assert np.array_equal(ranks, exp)


def _model(n, seed, cplx=False):
    rng = np.random.default_rng(seed)
    om = rng.uniform(0.5, 2.0, n) + (1j * rng.uniform(-0.5, 0.5, n) if cplx else 0)
    de = rng.uniform(-2, 2, n)
    pos = configs.chain_positions(n, a=5.5, jitter=rng.uniform(-0.5, 0.5, n))
    pairs = configs.pairs_from_positions(pos)
    return om, de, pairs


@pytest.mark.parametrize("name,n,edges,kind,k", GRAPHS)
@pytest.mark.parametrize("dtype", ["float64", "float32", "complex128", "complex64"])
def test_hv_matches_oracle(ctx, name, n, edges, kind, k, dtype):
    import torch
    from energy_level_b200.core import Basis, Hamiltonian
    cplx = dtype.startswith("complex")
    om, de, pairs = _model(n, 3, cplx=cplx)
    b = Basis(ctx, n, kind=kind, edges=edges, k=k)
    h = Hamiltonian(ctx, b, om, de, pairs)
    codes = None if kind == "full" else oracle_codes(n, edges, kind, k)
    rng = np.random.default_rng(1)
    for nvec in (1, 2, 4, 8, 32):
        x = rng.normal(size=(b.dim, nvec))
        if cplx:
            x = x + 1j * rng.normal(size=(b.dim, nvec))
        want = ref.hv(n, codes, om if cplx else om.real, de, pairs, x)
        tx = torch.as_tensor(x, dtype=getattr(torch, dtype), device=ctx.device)
        got = h.hv(tx).cpu().numpy()
        tol = 1e-12 if dtype in ("float64", "complex128") else 2e-5
        scale = max(1.0, np.abs(want).max())
        assert np.abs(got - want).max() <= tol * scale * 10, (dtype, nvec)


def test_diag_matches_oracle(ctx):
    from energy_level_b200.core import Basis, Hamiltonian
    n = 12
    om, de, pairs = _model(n, 4)
    edges = configs.chain_edges(n)
    b = Basis(ctx, n, kind="blockade", edges=edges)
    h = Hamiltonian(ctx, b, om.real, de, pairs)
    codes = ref.independent_states(n, edges, None)
    assert np.allclose(h.diag().cpu().numpy(), ref.diagonal(n, codes, de, pairs), atol=1e-12, rtol=0)
