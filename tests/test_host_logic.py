"""CPU tests of the host layer: backend declarations and routing rules,
model validation, state grammar, segment resolution, KPM post-processing."""
import os
import types

import numpy as np
import pytest

from energy_level_b200 import backends, configs, engine, kpm as bkpm, model
from energy_level_b200.state import state_vector
from oracle import ref

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_backend_names_and_capabilities():
    assert backends.normalize_equilibrium_backend("b200-lanczos", "gs") == "b200-lanczos"
    assert backends.normalize_equilibrium_backend("kpm-b200", "dos") == "b200-kpm"
    with pytest.raises(ValueError):
        backends.normalize_equilibrium_backend("b200-kpm", "gs")
    assert backends.normalize_time_backend("chebyshev-gpu") == "b200-cheb"
    b = backends.TIME_BACKENDS["b200-cheb"]
    assert b.segments and b.projected and b.return_state and b.gamma
    assert backends.engine_entries()[("b200-cheb", "many")] == ("energy_level_b200.engine", "evolve_manybody")


def test_capability_refusals_are_config_conflicts():
    # loss rates run on the non-Hermitian Taylor path
    backends.validate_time_capabilities("b200-cheb", gamma=[0.1, 0.0])
    with pytest.raises(model.ConfigConflict) as e:
        backends.validate_time_capabilities("b200-cheb", charge_sector=2)
    assert e.value.keys == ("manybody.charge_sector",)
    # Pauli strings are evaluated on the device ('full' capability, as the ed engine)
    backends.validate_time_capabilities("b200-cheb", pauli_strings=[{"label": "x"}])
    assert backends.TIME_BACKENDS["b200-cheb"].pauli == "full"
    with pytest.raises(ValueError):
        backends.validate_time_capabilities("b200-cheb", psi0="ground")
    backends.validate_time_capabilities("b200-cheb", segments=[{"t0": 0}], plan={"projected": True})


def test_install_into_reference_shaped_module():
    from dataclasses import dataclass

    @dataclass(frozen=True)
    class TimeBackend:
        module: str
        function: str
        aliases: tuple = ()
        options: tuple = ()
        segments: bool = False
        projected: bool = False
        gamma: bool = False
        return_state: bool = False

    fake = types.SimpleNamespace(EQ_BACKENDS={"ed": ("gs",)}, TIME_BACKENDS={}, TimeBackend=TimeBackend)
    backends.install_into(fake)
    assert fake.EQ_BACKENDS["b200-kpm"] == ("thermal", "dos")
    assert fake.TIME_BACKENDS["b200-cheb"].module == "b200_shim"
    assert fake.TIME_BACKENDS["b200-cheb"].projected


def test_install_into_the_reference_backends_module():
    """install_into on the reference's own backends.py (a fresh copy of the
    module), then the reference's validate_time_capabilities for b200-cheb:
    Pauli strings, drive segments, a projected plan, loss rates and
    return_state pass; a real-time charge sector is refused as for ed."""
    from conftest import reference_module
    rb = reference_module("src/core/manybody/backends.py", "_el_ref_backends")
    backends.install_into(rb)
    tb = rb.TIME_BACKENDS["b200-cheb"]
    assert isinstance(tb, rb.TimeBackend)
    ours = backends.TIME_BACKENDS["b200-cheb"]
    for f in ("segments", "projected", "gamma", "return_state", "charge", "order", "pauli",
              "native_state", "algorithm", "aliases", "options"):
        assert getattr(tb, f) == getattr(ours, f), f
    assert rb.normalize_time_backend("chebyshev-gpu") == "b200-cheb"
    assert "b200-cheb" in rb.pauli_backends()
    assert rb.normalize_equilibrium_backend("b200-kpm", "dos") == "b200-kpm"
    assert rb.normalize_equilibrium_backend("b200-lanczos", "spectrum") == "b200-lanczos"
    rb.validate_time_capabilities("b200-cheb", pauli_strings=[{"label": "zz", "terms": [(0, "z")]}],
                                  segments=[{"t0": 0.0}], plan={"projected": True},
                                  gamma=[0.1, 0.0], return_state=True, psi0="gggg")
    with pytest.raises(rb.ConfigConflict) as e:
        rb.validate_time_capabilities("b200-cheb", charge_sector=2)
    assert e.value.keys == ("manybody.charge_sector",)
    entries = rb.engine_entries()
    assert entries[("b200-cheb", "many")] == (".manybody.b200_shim", "evolve_manybody")


def test_b200_kpm_refuses_exact_trace():
    """exact=True asks for the dense spectral trace; b200-kpm refuses it
    before any work, like gpu-kpm (eq_route.py:446-447)."""
    system = {"calib": configs.calib_from_positions(configs.chain_positions(4)),
              "Om": np.ones(4), "delta": np.zeros(4)}
    for want in ("dos", "thermal"):
        with pytest.raises(ValueError, match="exact"):
            backends.solve_equilibrium(system, want, backend="b200-kpm", exact=True)


def test_model_refuses_unimplemented_channels():
    calib = configs.calib_from_positions(configs.chain_positions(4))
    n, om, de, pairs = model.model_arrays(calib, np.ones(4), np.zeros(4))
    assert n == 4 and len(pairs) == 6
    bad = dict(calib, terms=["I1", "I2"])
    bad["pairs"] = [dict(p, J=0.3) for p in calib["pairs"]]
    with pytest.raises(model.ConfigConflict):
        model.model_arrays(bad, np.ones(4), np.zeros(4))
    with pytest.raises(model.ConfigConflict):
        model.model_arrays(calib, np.ones(4), np.zeros(4), gamma=np.full(4, 0.1))
    with pytest.raises(ValueError):
        model.model_arrays(calib, np.ones(3), np.zeros(4))
    with pytest.raises(ValueError):
        model.model_arrays({"atoms": [], "pairs": []})


def test_model_columns_match_active_terms():
    """Without ``terms`` the channels in use are the calib's own (its 'terms'
    key, else every channel with a nonzero pair value), exactly as if
    active_terms(calib) had been passed; the column form equals the tuples."""
    calib = {k: v for k, v in configs.calib_from_positions(configs.chain_positions(5)).items()
             if k != "terms"}
    variants = [calib,
                dict(calib, pairs=[dict(p, V=0.0) for p in calib["pairs"]]),
                dict(calib, pairs=[dict(p, V=float("nan") if k == 0 else 0.0)
                                   for k, p in enumerate(calib["pairs"])]),
                dict(calib, pairs=[dict(p, J=0.0, A=None) for p in calib["pairs"]]),
                dict(calib, terms=["I1"], pairs=[dict(p, J=0.5) for p in calib["pairs"]])]
    for c in variants:
        ex_a, ex_b = [], []
        got = model.model_arrays(c, np.ones(5), np.zeros(5), exchange=ex_a)
        want = model.model_arrays(c, np.ones(5), np.zeros(5), terms=model.active_terms(c), exchange=ex_b)
        assert got[0] == want[0] and repr(got[3]) == repr(want[3]) and ex_a == ex_b
        n, _, _, (pi, pj, V) = model.model_columns(c, np.ones(5), np.zeros(5), exchange=[])
        assert repr(list(zip(pi.tolist(), pj.tolist(), V.tolist()))) == repr(got[3])
        assert pi.dtype == np.int32 and V.dtype == np.float64
    # numpy complex scalars keep their imaginary parts
    cj = dict(calib, terms=["I1", "I2"], pairs=[dict(p, J=np.complex128(0.5 + 0.25j)) for p in calib["pairs"]])
    ex = []
    model.model_columns(cj, np.ones(5), np.zeros(5), exchange=ex)
    assert ex and all(e[2] == 0.5 + 0.25j for e in ex)
    with pytest.raises(ValueError):
        model.model_columns(dict(calib, pairs=[dict(p, V=np.complex128(1 + 1j)) for p in calib["pairs"]]),
                            np.ones(5), np.zeros(5))
    with pytest.raises(model.ConfigConflict):   # J in use without an exchange list
        model.model_columns(dict(calib, pairs=[dict(p, J=0.5) for p in calib["pairs"]]),
                            np.ones(5), np.zeros(5))


def test_state_grammar_full_and_projected():
    n = 6
    codes = ref.independent_states(n, configs.chain_edges(n), None)
    v = state_vector("rgrgrg", n, codes)
    assert np.count_nonzero(v) == 1 and v[np.searchsorted(codes, 0b101010)] == 1
    full = state_vector(None, n)
    assert full[0] == 1 and np.linalg.norm(full) == pytest.approx(1.0)
    with pytest.raises(ValueError):
        state_vector("rrgggg", n, codes)     # weight outside the blockade basis
    sup = state_vector(("sup", [("gggggg", 1.0), ("rggggg", 1.0)]), n, codes)
    assert np.allclose(np.abs(sup[sup != 0]), 1 / np.sqrt(2))
    prod = state_vector([[1, 1]] * 2 + ["g"] * 4, 4 + 2)
    assert np.count_nonzero(prod) == 4


def test_segment_rules_match_oracle():
    n = 3
    segs = [{"t0": 0.0, "Om": [1, 1, 1], "delta": [0, 0, 0]},
            {"t0": 5.0, "Om": [2, 2, 2], "delta": [1, 1, 1], "phase": [0.5, 0, 0]}]
    assert engine.segment_intervals(0.0, 10.0, segs) == ref.segment_intervals(0.0, 10.0, segs)
    om, de = engine.segment_drive(7.0, segs, n)
    om2, de2 = ref.segment_drive(7.0, segs, n)
    assert np.allclose(om, om2) and np.allclose(de, de2)
    om3, de3 = engine.segment_drive(2.0, segs, n, interp="midpoint")
    assert np.allclose(om3, 0.5 * (np.ones(3) + 2.0 * np.exp(1j * np.array([0.5, 0.0, 0.0]))))
    assert np.allclose(de3, 0.5)
    with pytest.raises(ValueError):
        engine.time_grid([0.0])
    with pytest.raises(RuntimeError, match="用户取消"):
        engine.check_cancel(np.array([0.0, 1.0]))


def test_kpm_postprocessing_matches_reference_golden():
    g = np.load(os.path.join(GOLD, "kpm.npz"))
    num = int(g["num"])
    assert np.max(np.abs(bkpm.jackson_kernel(num) - g["jackson"])) < 1e-15
    rho = bkpm.dos_from_moments(g["mu"], float(g["c"]), float(g["r"]), g["energies"], num)
    assert np.max(np.abs(rho - g["rho"])) < 1e-12
    c, r = bkpm.kpm_scale(float(g["emin"]), float(g["emax"]))
    assert abs(c - float(g["c"])) < 1e-12 and abs(r - float(g["r"])) < 1e-12


def test_kpm_thermal_from_exact_moments_matches_spectrum():
    g = np.load(os.path.join(GOLD, "kpm.npz"))
    n = int(g["n"])
    H = ref.dense_h(n, None, g["om"], g["de"], [(int(i), int(j), v) for i, j, v in g["pairs"]])
    w = np.linalg.eigvalsh(H)
    c, r = float(g["c"]), float(g["r"])
    mu = ref.kpm_moments_exact(H, 512, c, r)
    th = bkpm.thermal_from_moments(len(w), [0.1, 0.5], (mu, c, r), 512)
    for i, b in enumerate([0.1, 0.5]):
        p = np.exp(-b * (w - w.min()))
        E = float(p @ w / p.sum())
        assert abs(th["E"][i] - E) < 1e-5


def test_exchange_parsing_and_number_conservation():
    xy = configs.xy_chain(6)
    ex = []
    n, om, de, pairs = model.model_arrays(xy["calib"], xy["Om"], xy["delta"], terms=["I1", "I2"], exchange=ex)
    assert n == 6 and len(pairs) == 15 and len(ex) == 15
    assert all(e[3] == 0 for e in ex) and all(e[2] != 0 for e in ex)
    # without an exchange list a nonzero J is refused, never dropped
    with pytest.raises(model.ConfigConflict):
        model.model_arrays(xy["calib"], xy["Om"], xy["delta"], terms=["I1", "I2"])
    # I2 not among the terms: J is ignored as in channels.py
    ex2 = []
    model.model_arrays(xy["calib"], xy["Om"], xy["delta"], terms=["I1"], exchange=ex2)
    assert ex2 == []
    model.check_number_conserving(xy["calib"], np.zeros(6), ["I1", "I2"])
    with pytest.raises(ValueError):
        model.check_number_conserving(xy["calib"], np.full(6, 0.1), ["I1", "I2"])
    cal = dict(xy["calib"], pairs=[dict(p, A=0.2) for p in xy["calib"]["pairs"]])
    with pytest.raises(ValueError):
        model.check_number_conserving(cal, np.zeros(6), ["I1", "I2", "I3"])
    # loss rates: refused unless the caller propagates in time
    with pytest.raises(model.ConfigConflict):
        model.model_arrays(xy["calib"], xy["Om"], xy["delta"], gamma=np.full(6, 0.1), terms=["I1"])
    model.model_arrays(xy["calib"], xy["Om"], xy["delta"], gamma=np.full(6, 0.1), terms=["I1"], allow_loss=True)


def test_sector_scan_refuses_before_touching_the_device():
    from energy_level_b200.sector_scan import SectorScan, scan_ground_sectors
    xy = configs.xy_chain(6)
    with pytest.raises(ValueError):
        SectorScan(xy["calib"], xy["delta"], np.full(6, 0.1), terms=["I1", "I2"])
    with pytest.raises(ValueError):
        SectorScan(xy["calib"], xy["delta"], np.zeros(6), terms=["I1", "I2"], sectors=[0, 7])
    with pytest.raises(ValueError):
        SectorScan(xy["calib"], xy["delta"], np.zeros(6), gamma=np.full(6, 0.1))
    with pytest.raises(ValueError):
        scan_ground_sectors(xy["calib"], xy["delta"], np.zeros(6), terms=["I1", "I2"], backend="dmrg")
    with pytest.raises(ValueError):
        SectorScan({"atoms": [], "pairs": []})


def test_pack_instances_matches_calib_pairs():
    """The batched solver's host arrays, against a direct walk over each
    instance's calib: sizes, layouts, drive columns and the V pairs in calib
    order with their offsets; an instance without pairs adds none."""
    from energy_level_b200 import _lib, batched
    insts = configs.batch512(count=24, seed=4)
    lone = {"atoms": [{"id": 0, "pos": [0.0, 0.0, 0.0]}, {"id": 1, "pos": [9.0, 0.0, 0.0]}],
            "pairs": [], "terms": ["I1"]}
    insts.append(dict(calib=lone, Om=np.full(2, 2.0), delta=np.zeros(2), edges=None))
    k = batched.pack_instances(insts)
    assert [a.dtype for a in k] == [np.int32, np.int32, np.float64, np.float64,
                                    np.int32, np.int32, np.int32, np.float64,
                                    np.int32, np.int32, np.int32]
    assert k[0].tolist() == [len(i["calib"]["atoms"]) for i in insts]
    assert k[1].tolist() == [_lib.EL_LAYOUT_CHAIN] * 24 + [_lib.EL_LAYOUT_FULL]
    eoff = [0]
    for inst in insts:
        eoff.append(eoff[-1] + len(inst["edges"] or []))
    assert k[8].tolist() == eoff
    assert np.array_equal(k[2], np.concatenate([np.asarray(i["Om"], float) for i in insts]))
    assert np.array_equal(k[3], np.concatenate([np.asarray(i["delta"], float) for i in insts]))
    offs, pi, pj, V = [0], [], [], []
    for inst in insts:
        for p in inst["calib"]["pairs"]:
            if p.get("V"):
                pi.append(p["i"]); pj.append(p["j"]); V.append(p["V"])
        offs.append(len(V))
    assert k[4].tolist() == offs and offs[-1] == offs[-2]
    assert k[5].tolist() == pi and k[6].tolist() == pj and k[7].tolist() == V
    empty = batched.pack_instances([dict(calib=lone, Om=np.ones(2), delta=np.zeros(2), edges=None)])
    assert empty[4].tolist() == [0, 0] and empty[5].tolist() == [0] and empty[7].tolist() == [0.0]
    with pytest.raises(ValueError):
        batched.pack_instances([dict(calib=lone, Om=np.array([1j, 0]), delta=np.zeros(2), edges=None)])


def test_batched_layout_of_each_blockade_graph():
    """A path or cycle keeps the arithmetic layouts, any other graph becomes
    a code table (its edges normalised and passed on), no edges the full
    basis; an edge outside the instance is refused on the host."""
    from energy_level_b200 import _lib, batched
    assert batched._layout(5, None) == (_lib.EL_LAYOUT_FULL, [])
    assert batched._layout(5, [(1, 2), (0, 1), (3, 2), (3, 4)])[0] == _lib.EL_LAYOUT_CHAIN
    assert batched._layout(5, [(0, 1), (1, 2), (2, 3), (3, 4), (4, 0)])[0] == _lib.EL_LAYOUT_RING
    lay, es = batched._layout(4, [(1, 0), (0, 2), (2, 1), (3, 2)])
    assert lay == _lib.EL_LAYOUT_TABLE and es == [(0, 1), (0, 2), (1, 2), (2, 3)]
    with pytest.raises(ValueError):
        batched._layout(4, [(0, 4)])
    with pytest.raises(ValueError):
        batched._layout(4, [(2, 2)])
    star = {"atoms": [{"id": i, "pos": p} for i, p in enumerate([[0.0, 0.0, 0.0], [6.0, 0.0, 0.0],
                                                                  [0.0, 6.0, 0.0], [-6.0, 0.0, 0.0]])],
            "pairs": [], "terms": ["I1"]}
    k = batched.pack_instances([dict(calib=star, Om=np.ones(4), delta=np.zeros(4),
                                     edges=[(0, 1), (0, 2), (3, 0)])])
    assert k[1].tolist() == [_lib.EL_LAYOUT_TABLE]
    assert k[8].tolist() == [0, 3] and k[9].tolist() == [0, 0, 0] and k[10].tolist() == [1, 2, 3]


def test_pulse_problem_refuses_exchange_channels():
    """The adjoint differentiates the Omega/delta/V model: J or A in use is a
    ConfigConflict, raised on the host before any device work."""
    from energy_level_b200.adjoint import PulseProblem
    xy = configs.xy_chain(6, seed=2)
    with pytest.raises(model.ConfigConflict):
        PulseProblem(dict(xy["calib"], terms=["I1", "I2"]), "g" * 6, target="rgrgrg")


def test_segment_table_equals_segment_drive():
    """The evolution loop's pre-sorted segment table returns exactly the
    drive of segment_drive (runtime.py:90-114) at every time, ties and
    unsorted t0 included, for both interpolation rules."""
    rng = np.random.default_rng(11)
    n = 4
    t0s = [5.0, 0.0, 2.5, 2.5, 9.0, 7.25]
    segs = [{"t0": t0, "Om": rng.uniform(0, 3, n), "delta": rng.uniform(-2, 2, n),
             "phase": rng.uniform(-1, 1, n)} for t0 in t0s]
    table = engine.SegmentTable(segs, n)
    times = [-1.0, 0.0, 1.0, 2.5, 3.0, 5.0, 7.25, 8.0, 9.0, 12.0] + list(rng.uniform(-1, 12, 40))
    for interp in ("left", "midpoint"):
        for t in times:
            om, de = engine.segment_drive(t, segs, n, interp=interp)
            om2, de2 = table.drive(t, interp=interp)
            assert np.array_equal(om, om2) and np.array_equal(de, de2), (interp, t)
    with pytest.raises(ValueError):
        table.drive(1.0, interp="cubic")


class _NoLaunchContext:
    """Stands in for a library context: any call through it fails the test,
    so a refusal is shown to happen before a device address is passed on."""

    def __init__(self):
        import torch
        self.device = torch.device("cuda", 0)

    def call(self, name, *args):
        raise AssertionError("%s reached the library" % name)


@pytest.mark.parametrize("wrapper", ["cheb_step", "taylor_step", "observables", "observables_noalloc",
                                     "spin_observables", "pauli_expect"])
def test_state_wrappers_refuse_bad_vectors_before_any_call(wrapper):
    """Every wrapper that hands a state's address to the library refuses a
    vector of the wrong length, a non-contiguous view and a host tensor with
    ValueError, without calling the library."""
    import torch
    from energy_level_b200 import solvers
    ham = types.SimpleNamespace(ctx=_NoLaunchContext(), dim=16, n=4, handle=None)
    args = {"cheb_step": (1.0,), "taylor_step": (1.0,), "spin_observables": ((),),
            "pauli_expect": ([{"label": "z", "terms": [(0, "z")]}],)}.get(wrapper, ())
    fn = getattr(solvers, wrapper)
    short = torch.zeros(15, dtype=torch.complex64)
    host = torch.zeros(16, dtype=torch.complex64)
    strided = torch.zeros(32, dtype=torch.complex64)[::2]
    for bad in (short, host) + ((strided,) if wrapper in ("cheb_step", "taylor_step", "observables_noalloc") else ()):
        with pytest.raises(ValueError):
            fn(ham, bad, *args)
    if wrapper in ("cheb_step", "taylor_step"):
        with pytest.raises(ValueError):
            fn(ham, torch.zeros(16, dtype=torch.float32), *args)


def test_hv_refuses_host_and_short_vectors():
    import torch
    from energy_level_b200.core import Hamiltonian
    ham = Hamiltonian.__new__(Hamiltonian)
    ham.ctx, ham.dim, ham.handle = _NoLaunchContext(), 16, None
    for bad in (torch.zeros(15), torch.zeros(16), torch.zeros(16, 3, dtype=torch.int32)):
        with pytest.raises(ValueError):
            ham.hv(bad)


def _constraint_gold():
    import json
    g = np.load(os.path.join(GOLD, "constraint.npz"))
    calib = configs.calib_from_positions(g["pos"])
    return g, calib, [(str(nm), json.loads(str(g[str(nm) + "_spec"]))) for nm in g["names"]]


def test_constraint_specs_resolve_like_build_plan():
    """Edges and projection of blockade / pxp specs with threshold_mhz,
    'auto' edges and mode='full' equal the reference's build_plan
    (hamiltonian_plan.py:15-72) on a 3x4 lattice; a projecting spec with
    neither edges nor a threshold is refused."""
    g, calib, specs = _constraint_gold()
    for name, spec in specs:
        projected, edges, norm = model.resolve_constraint(calib, spec)
        assert projected == bool(g[name + "_projected"]), name
        assert np.array_equal(np.asarray(edges, np.int64).reshape(-1, 2), g[name + "_edges"]), name
    with pytest.raises(ValueError, match="threshold_mhz"):
        model.resolve_constraint(calib, {"kind": "blockade"})
    assert str(g["refusal"]).startswith("blockade/PXP project")
    with pytest.raises(ValueError):
        model.resolve_constraint(calib, "pxp")
    with pytest.raises(ValueError):
        model.resolve_constraint(calib, {"kind": "rydberg"})
    with pytest.raises(ValueError):
        model.resolve_constraint(calib, {"kind": "blockade", "edges": [[0, 0]]})
    with pytest.raises(ValueError):
        model.resolve_constraint(calib, {"kind": "blockade", "edges": "nearest"})
    assert model.resolve_constraint(calib, None)[0] is False
    assert model.resolve_constraint(calib, {"kind": "blockade", "edges": [[3, 1], [1, 3]]})[1] == [[1, 3]]
    # a projected plan without edges takes them from its spec, or is refused
    assert model.plan_edges({"projected": True, "constraint": specs[0][1], "calib": calib}) == \
        g[specs[0][0] + "_edges"].tolist()
    with pytest.raises(ValueError):
        model.plan_edges({"projected": True})
