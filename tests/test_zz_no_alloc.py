"""el_observables_noalloc against el_observables.

The no-allocation entry point keeps its reduction scratch in a static device
array; these tests run it twice in a row on the same and on different states
and compare each result with el_observables (same sums, other block count,
so within 1e-12 relative).  The file is collected last so that it also runs
after every other GPU test in one session."""
import numpy as np
import pytest

from energy_level_b200 import configs, model, solvers
from energy_level_b200.core import Basis, Hamiltonian

pytestmark = pytest.mark.gpu

MAX_SITES = 40


def _random_state(torch, dim, dtype, seed):
    g = torch.Generator(device='cpu').manual_seed(seed)
    if dtype.is_complex:
        re = torch.randn(dim, generator=g, dtype=torch.float64)
        im = torch.randn(dim, generator=g, dtype=torch.float64)
        v = torch.complex(re, im)
    else:
        v = torch.randn(dim, generator=g, dtype=torch.float64)
    return (v / v.abs().pow(2).sum().sqrt()).to(dtype).cuda()


def _compare(ham, psi):
    ns_ref, nrm_ref = solvers.observables(ham, psi)
    ns, nrm = solvers.observables_noalloc(ham, psi)
    assert abs(nrm - nrm_ref) <= 1e-12 * max(1.0, abs(nrm_ref))
    assert np.max(np.abs(ns - ns_ref)) <= 1e-12 * max(1.0, np.max(np.abs(ns_ref)))
    return ns, nrm


@pytest.mark.parametrize('dtype', ['float32', 'float64', 'complex64', 'complex128'])
def test_ring_blockade_two_calls(ctx, dtype):
    import torch
    n = 20
    calib = configs.calib_from_positions(configs.ring_positions(n))
    plan = {'projected': True, 'blockade_edges': configs.ring_edges(n), 'constraint': {'kind': 'blockade'}}
    _, basis, ham, _ = model.build(calib, np.full(n, 2.0), np.zeros(n), plan=plan)
    td = getattr(torch, dtype)
    a = _random_state(torch, basis.dim, td, 1)
    b = _random_state(torch, basis.dim, td, 2)
    first = _compare(ham, a)
    second = _compare(ham, a)          # same state again: scratch reused
    assert np.array_equal(first[0], second[0]) and first[1] == second[1]
    _compare(ham, b)                   # different state right after


def test_full_basis_grid_stride(ctx):
    """dim = 2^24 rows > 592 blocks x 256 threads: every block strides."""
    import torch
    n = 24
    basis = Basis(ctx, n, 'full')
    ham = Hamiltonian(ctx, basis, np.ones(n), np.zeros(n), [])
    psi = _random_state(torch, basis.dim, torch.complex64, 3)
    for _ in range(2):
        _compare(ham, psi)


def test_site_limit(ctx):
    """40 sites (the limit) works; 41 sites are refused with a message."""
    import torch
    for n, ok in ((MAX_SITES, True), (MAX_SITES + 1, False)):
        basis = Basis(ctx, n, 'charge', k=2)
        ham = Hamiltonian(ctx, basis, np.zeros(n), np.zeros(n), [])
        psi = _random_state(torch, basis.dim, torch.float64, 4)
        if ok:
            _compare(ham, psi)
        else:
            with pytest.raises(ValueError, match='static scratch limit of 40 sites'):
                solvers.observables_noalloc(ham, psi)
            solvers.observables(ham, psi)   # the allocating entry point still serves it


def test_no_device_memory_change(ctx):
    """After the first call on the device, calls leave free device memory unchanged."""
    import torch
    n = 16
    basis = Basis(ctx, n, 'full')
    ham = Hamiltonian(ctx, basis, np.ones(n), np.zeros(n), [])
    psi = _random_state(torch, basis.dim, torch.complex128, 5)
    solvers.observables_noalloc(ham, psi)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        solvers.observables_noalloc(ham, psi)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
