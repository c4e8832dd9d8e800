"""GPU parity of the batched ground-state solvers on blockade sectors of
arbitrary graphs (the TABLE layout: 2-D lattices with nearest-neighbour and
diagonal blockade, a random graph), mixed with chain, ring and full-basis
instances in one batch, against dense eigenpairs from the oracle — the
batched ground state of the reference (equilibrium.py:251-311) on plans of
any constraint graph (hamiltonian_plan.py:15-50)."""
import numpy as np
import pytest

from oracle import ref
from energy_level_b200 import configs

pytestmark = pytest.mark.gpu


def _lattice(nx, ny, a=6.0):
    return [[a * x, a * y, 0.0] for y in range(ny) for x in range(nx)]


def _edges_within(pos, r):
    pos = np.asarray(pos, float)
    n = len(pos)
    return [(i, j) for i in range(n) for j in range(i + 1, n) if np.linalg.norm(pos[i] - pos[j]) <= r]


def _instances(seed=21):
    rng = np.random.default_rng(seed)
    out = []
    specs = [
        ("lattice", (3, 3), 6.1),     # nearest-neighbour blockade
        ("lattice", (3, 4), 8.6),     # with the diagonals
        ("lattice", (4, 4), 6.1),
        ("random", 11, None),
        ("chain", 13, None),
        ("ring", 10, None),
        ("full", 9, None),
        ("lattice", (2, 5), 8.6),
    ]
    for kind, size, r in specs:
        if kind == "lattice":
            pos = _lattice(*size)
            edges = _edges_within(pos, r)
        elif kind == "random":
            pos = [[6.0 * i, 0.0, 0.0] for i in range(size)]
            edges = [(i, j) for i in range(size) for j in range(i + 1, size) if rng.random() < 0.25]
        else:
            pos = configs.chain_positions(size, jitter=rng.uniform(-0.3, 0.3, size))
            edges = {"chain": configs.chain_edges(size), "ring": configs.ring_edges(size), "full": None}[kind]
        n = len(pos)
        calib = configs.calib_from_positions(pos)
        om, de = rng.uniform(1.5, 2.5, n), rng.uniform(-3.0, 1.0, n)
        out.append(dict(calib=calib, Om=om, delta=de, edges=edges))
    return out


def _dense(inst):
    n = len(inst["Om"])
    codes = None if inst["edges"] is None else ref.independent_states(n, inst["edges"], None)
    pairs = [(p["i"], p["j"], p["V"]) for p in inst["calib"]["pairs"]]
    w, v = np.linalg.eigh(ref.dense_h(n, codes, inst["Om"], inst["delta"], pairs))
    return w[0], w[1] - w[0], ref.site_occupations(n, codes, v[:, 0])


@pytest.mark.parametrize("mode", ["batch", "coop"])
def test_graph_blockade_batch_matches_dense(ctx, mode):
    from energy_level_b200 import _lib
    from energy_level_b200.batched import batched_ground_states, pack_instances
    insts = _instances()
    lays = pack_instances(insts)[1].tolist()
    assert lays.count(_lib.EL_LAYOUT_TABLE) == 5
    out = batched_ground_states(insts, dtype="float64", max_iter=300, tol=1e-11, mode=mode)
    assert out["mode"] == mode and out["converged"].all()
    for i, inst in enumerate(insts):
        e0, gap, occ = _dense(inst)
        n = len(inst["Om"])
        assert abs(out["E0"][i] - e0) < 1e-9 * max(1.0, abs(e0)), i
        assert abs(out["gap"][i] - gap) < 1e-7, i
        assert np.max(np.abs(out["n_atom"][i, :n] - occ)) < 1e-7, i


def test_graph_blockade_batch_fp32(ctx):
    from energy_level_b200.batched import BatchedGroundStates
    insts = _instances(seed=5)
    b = BatchedGroundStates(insts, dtype="float32", max_iter=300, tol=1e-5)
    b.run()
    r = b.results()
    assert r["converged"].all()
    for i, inst in enumerate(insts):
        e0, gap, _ = _dense(inst)
        assert abs(r["E0"][i] - e0) < 2e-6 * max(1.0, abs(e0)), i
    # the same batch again: same bits (fixed-order reductions)
    b.run()
    assert np.array_equal(b.results()["E0"], r["E0"])
    b.close()


def test_graph_blockade_needs_edges_and_a_bounded_sector(ctx):
    """A TABLE instance without edges, and a graph whose blockade sector
    exceeds 2^24 rows, are refused by the library before any device work."""
    import ctypes as C
    from energy_level_b200 import _lib
    ns = np.array([4], np.int32)
    lay = np.array([_lib.EL_LAYOUT_TABLE], np.int32)
    om, de = np.ones(4), np.zeros(4)
    poff = np.zeros(2, np.int32)
    dummy_i, dummy_v = np.zeros(1, np.int32), np.zeros(1)
    h = C.c_void_p()
    lib = ctx.lib
    rc = lib.el_batch_create_graph(ctx.handle, 1, ns.ctypes.data, lay.ctypes.data, _lib.dptr(om), _lib.dptr(de),
                                   poff.ctypes.data, dummy_i.ctypes.data, dummy_i.ctypes.data, _lib.dptr(dummy_v),
                                   None, None, None, _lib.EL_F64, 100, 1e-10, C.byref(h))
    assert rc == _lib.EL_EINVAL and not h.value
    n = 40                                  # no edge but one: ~2^40 rows
    ns = np.array([n], np.int32)
    om, de = np.ones(n), np.zeros(n)
    eoff = np.array([0, 1], np.int32)
    ea, eb = np.array([0], np.int32), np.array([1], np.int32)
    rc = lib.el_batch_create_graph(ctx.handle, 1, ns.ctypes.data, lay.ctypes.data, _lib.dptr(om), _lib.dptr(de),
                                   poff.ctypes.data, dummy_i.ctypes.data, dummy_i.ctypes.data, _lib.dptr(dummy_v),
                                   eoff.ctypes.data, ea.ctypes.data, eb.ctypes.data, _lib.EL_F64, 100, 1e-10,
                                   C.byref(h))
    assert rc == _lib.EL_EINVAL and not h.value
