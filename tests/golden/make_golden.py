"""Generate golden fixtures by running the energy-level reference itself.

Run in a checkout where the reference tree is importable:

    python tests/golden/make_golden.py /path/to/energy-level

It writes small .npz files next to this script.  The GPU tests, the CPU
oracle tests and smoke() compare against these files; nothing at test time
imports the reference.  Every call below is a public function of the
reference's src/core/manybody package (file:line given per fixture).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root: str) -> None:
    sys.path.insert(0, ref_root)
    from src.core.manybody import basis as rbasis                       # basis.py
    from src.core.manybody import matrix_free as rmf                    # matrix_free.py
    from src.core.manybody import assemble as rasm                      # assemble.py
    from src.core.manybody import kpm as rkpm                           # kpm.py
    from src.core.manybody import equilibrium as req                    # equilibrium.py
    from src.core.manybody import engine_ed as red                      # engine_ed.py
    from src.core.manybody import hamiltonian_plan as rplan             # hamiltonian_plan.py

    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from energy_level_b200 import configs

    # -- basis codes: independent_states (basis.py:24-47), number_sector_basis
    #    (matrix_free.py:12-38), independent_set_count (basis.py:50-76)
    graphs = {
        "chain10": (10, configs.chain_edges(10)),
        "ring11": (11, configs.ring_edges(11)),
        "ring20": (20, configs.ring_edges(20)),
        "square3x3": (9, [[0, 1], [1, 2], [3, 4], [4, 5], [6, 7], [7, 8], [0, 3], [3, 6],
                          [1, 4], [4, 7], [2, 5], [5, 8]]),
        "nnn_chain12": (12, configs.chain_edges(12) + [[i, i + 2] for i in range(10)]),
        "chain22": (22, configs.chain_edges(22)),
    }
    out = {}
    for name, (n, edges) in graphs.items():
        codes = np.asarray(rbasis.independent_states(n, edges, max_states=1 << 22), np.int64)
        out["codes_" + name] = codes
        out["edges_" + name] = np.asarray(edges, np.int64)
        out["n_" + name] = np.int64(n)
        out["count_" + name] = np.int64(rbasis.independent_set_count(n, edges))
    for n, k in [(10, 4), (12, 6), (6, 0), (6, 6)]:
        out["charge_%d_%d" % (n, k)] = np.asarray(rmf.number_sector_basis(n, k), np.int64)
    np.savez_compressed(os.path.join(HERE, "basis.npz"), **out)

    # -- H x: hamiltonian_linear_operator (matrix_free.py:51-62) on the full
    #    basis and on restricted bases; build_H_sparse diagonal (assemble.py:277)
    out = {}
    rng = np.random.default_rng(20261203)
    cases = {
        "full7": (7, None),
        "chain10": (10, configs.chain_edges(10)),
        "ring9": (9, configs.ring_edges(9)),
        "square3x3": (9, graphs["square3x3"][1]),
    }
    for name, (n, edges) in cases.items():
        pos = configs.chain_positions(n, a=5.5, jitter=rng.uniform(-0.4, 0.4, n))
        calib = configs.calib_from_positions(pos)
        om = rng.uniform(0.5, 2.5, n)
        de = rng.uniform(-3.0, 3.0, n)
        basis = None if edges is None else rbasis.independent_states(n, edges)
        op = rmf.hamiltonian_linear_operator(calib, Om=om, delta=de, terms=["I1"],
                                             basis_indices=basis)
        dim = op.shape[0]
        x = rng.normal(size=dim) + 1j * rng.normal(size=dim)
        out["x_" + name] = x
        out["y_" + name] = op @ x
        out["om_" + name] = om
        out["de_" + name] = de
        out["pairs_" + name] = np.asarray([[p["i"], p["j"], p["V"]] for p in calib["pairs"]])
        out["n_" + name] = np.int64(n)
        out["edges_" + name] = np.asarray(edges if edges else np.zeros((0, 2)), np.int64)
        H = rasm.build_H_sparse(calib, om, de, ["I1"], None, basis_indices=basis)
        out["diag_" + name] = np.asarray(H.diagonal()).real
    # complex Omega (phase) on a restricted basis: conj direction of channels.py:114-118
    n = 8
    pos = configs.chain_positions(n)
    calib = configs.calib_from_positions(pos)
    omc = rng.uniform(0.5, 2.0, n) * np.exp(1j * rng.uniform(0, 2 * np.pi, n))
    de = rng.uniform(-2, 2, n)
    basis = rbasis.independent_states(n, configs.chain_edges(n))
    op = rmf.hamiltonian_linear_operator(calib, Om=omc, delta=de, terms=["I1"], basis_indices=basis)
    x = rng.normal(size=len(basis)) + 1j * rng.normal(size=len(basis))
    out.update(x_cplx8=x, y_cplx8=op @ x, om_cplx8=omc, de_cplx8=de, n_cplx8=np.int64(n),
               pairs_cplx8=np.asarray([[p["i"], p["j"], p["V"]] for p in calib["pairs"]]),
               edges_cplx8=np.asarray(configs.chain_edges(n), np.int64))
    np.savez_compressed(os.path.join(HERE, "hv.npz"), **out)

    # -- KPM: kpm_moments (kpm.py:115-151) with its own numpy probe stream,
    #    exact moments, _bounds, jackson_kernel, _dos_from_moments
    n = 7
    pos = configs.chain_positions(n, a=5.5, jitter=rng.uniform(-0.4, 0.4, n))
    calib = configs.calib_from_positions(pos)
    om = rng.uniform(0.5, 2.0, n)
    de = rng.uniform(-3, 3, n)
    H = rasm.build_H_sparse(calib, om, de, ["I1"], None)
    num, nvec, seed = 48, 4, 3
    mu, c, r = rkpm.kpm_moments(H, num=num, nvec=nvec, seed=seed)
    probe_rng = np.random.default_rng(seed)
    z = np.stack([probe_rng.choice(np.array([-1.0, 1.0]), size=H.shape[0]) for _ in range(nvec)])
    mu_exact, _, _ = rkpm.kpm_moments(H, num=num, exact=True)
    emin, emax, c2, r2 = rkpm._bounds(H)
    energies = np.linspace(emin, emax, 64)
    rho = rkpm._dos_from_moments(mu, c, r, energies, num)
    np.savez_compressed(os.path.join(HERE, "kpm.npz"), n=np.int64(n), om=om, de=de,
                        pairs=np.asarray([[p["i"], p["j"], p["V"]] for p in calib["pairs"]]),
                        num=np.int64(num), nvec=np.int64(nvec), seed=np.int64(seed), mu=mu, c=c, r=r,
                        probes=z, mu_exact=mu_exact, emin=emin, emax=emax,
                        jackson=rkpm.jackson_kernel(num), energies=energies, rho=rho)

    # -- ground states: ground_state (equilibrium.py:35-96) with eigsh on the
    #    matrix-free operator for the chain12 workload; blockade sector by
    #    dense eigh of the projected plan (hamiltonian_plan.py:129-156)
    cfg = configs.chain12()
    op = rmf.hamiltonian_linear_operator(cfg["calib"], Om=cfg["Om"], delta=cfg["delta"], terms=["I1"])
    v0 = np.random.default_rng(0).standard_normal(op.shape[0])
    gs = req.ground_state(op, dense_max=0, k=2, v0=v0)
    plan = rplan.build_plan(cfg["calib"], Om=cfg["Om"], delta=cfg["delta"], terms=["I1"],
                            constraint={"kind": "blockade", "edges": configs.chain_edges(12)})
    gsb = req.ground_state(rplan.compile_sparse(plan), dense_max=4096, k=2)
    cfgr = configs.ring20()
    ring_pairs = np.asarray([[p["i"], p["j"], p["V"]] for p in cfgr["calib"]["pairs"]])
    plan_r = rplan.build_plan(cfgr["calib"], Om=np.full(20, 2.0), delta=np.full(20, 1.0),
                              terms=["I1"], constraint={"kind": "blockade", "edges": configs.ring_edges(20)})
    gsr = req.ground_state(rplan.compile_sparse(plan_r), dense_max=0, k=2,
                           v0=np.random.default_rng(1).standard_normal(plan_r["dim"]))
    np.savez_compressed(os.path.join(HERE, "ground.npz"),
                        chain12_E0=gs["E0"], chain12_gap=gs["gap"], chain12_evals=gs["evals"],
                        chain12b_E0=gsb["E0"], chain12b_gap=gsb["gap"],
                        ring20_E0=gsr["E0"], ring20_gap=gsr["gap"], ring20_pairs=ring_pairs)

    # -- evolution: evolve_manybody (engine_ed.py:153-372) with piecewise-
    #    constant segments on a projected blockade plan (segment path,
    #    engine_ed.py:130-147), record_psi for the final state
    n = 9
    calib = configs.calib_from_positions(configs.chain_positions(n))
    steps, total = 12, 240.0
    segments = [{"t0": k * total / steps, "Om": np.full(n, 2.0 + 0.3 * np.sin(k)),
                 "delta": np.full(n, 6.0 - 12.0 * k / steps)} for k in range(steps)]
    plan = rplan.build_plan(calib, Om=np.full(n, 2.0), delta=np.zeros(n), terms=["I1"],
                            constraint={"kind": "blockade", "edges": configs.chain_edges(n)})
    t_grid = np.linspace(0.0, total, 5)
    res = red.evolve_manybody(calib, psi0="g" * n, t_grid=t_grid, segments=segments, plan=plan,
                              terms=["I1"], record_psi=True, want_corr=False, want_entropy=False,
                              want_observables=False)
    np.savez_compressed(os.path.join(HERE, "evolve.npz"), n=np.int64(n), t_grid=t_grid,
                        seg_t0=np.asarray([s["t0"] for s in segments]),
                        seg_om=np.asarray([s["Om"] for s in segments]),
                        seg_de=np.asarray([s["delta"] for s in segments]),
                        pairs=np.asarray([[p["i"], p["j"], p["V"]] for p in calib["pairs"]]),
                        pops_atom=res["pops_atom"], norms=res["norms"], psi_final=res["psi_amp"],
                        basis_states=np.asarray(res["basis_states"], np.int64))
    print("golden fixtures written to", HERE)


def spectrum_fixture(ref_root: str) -> None:
    """Source-state spectrum: eq_route.solve_equilibrium(want='spectrum')
    (eq_route.py:260-337) with a site-weight source minus its mean, and the
    Lanczos tridiagonal of spectrum.lanczos (spectrum.py:34-103) from the same
    source state, on a 10-site chain blockade plan."""
    sys.path.insert(0, ref_root)
    from src.core.manybody import eq_route as rroute                    # eq_route.py
    from src.core.manybody import spectrum as rspec                     # spectrum.py
    from src.core.manybody import matrix_free as rmf                    # matrix_free.py
    from src.core.manybody import hamiltonian_plan as rplan             # hamiltonian_plan.py
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from energy_level_b200 import configs
    n = 10
    calib = configs.calib_from_positions(configs.chain_positions(n))
    om, de = np.full(n, 2.0), np.full(n, -1.5)
    plan = rplan.build_plan(calib, Om=om, delta=de, terms=["I1"],
                            constraint={"kind": "blockade", "edges": configs.chain_edges(n)})
    codes = np.asarray(plan["states"], np.int64)
    weights = np.cos(np.pi * np.arange(n) / 3.0)
    source = {"kind": "site_weights", "weights": weights, "subtract_mean": True}
    opts = {"eta": 0.1, "n_krylov": 40, "n_omega": 300}
    # the route on the full 2^N basis (the reference's spectrum route takes no
    # projected plan: its |0> and H live on the full space)
    sysd = {"calib": calib, "Om": om, "delta": de, "terms": ["I1"],
            "source": source, "spectrum": opts}
    try:
        res = rroute.solve_equilibrium(sysd, want="spectrum", backend="lanczos")
    except Exception as exc:   # route unavailable for this plan: keep the Lanczos part only
        print("spectrum route:", exc)
        res = None
    H = rmf.hamiltonian_linear_operator(calib, om, de, None, ["I1"], basis_indices=codes)
    rng = np.random.default_rng(7)
    psi = rng.normal(size=len(codes)) + 1j * rng.normal(size=len(codes))
    psi /= np.linalg.norm(psi)
    bits = np.asarray([((codes >> (n - 1 - i)) & 1) for i in range(n)], float)
    d = bits.T @ weights
    phi = d * psi
    lz = rspec.lanczos(H, phi, 40)
    sp = rspec.source_spectrum(H, phi, shift=0.3, eta=0.1, n_krylov=40, n_omega=300)
    out = dict(n=np.int64(n), om=om, de=de, codes=codes, weights=weights,
               pairs=np.asarray([[p["i"], p["j"], p["V"]] for p in calib["pairs"]]),
               psi=psi, phi=phi, alphas=lz["alphas"], betas=lz["betas"], norm2=lz["norm2"],
               lz_n=np.int64(lz["n"]), sp_omega=sp["omega"], sp_spectral=sp["spectral"],
               sp_evals=sp["evals"], sp_weights=sp["spectrum_weights"])
    if res is not None:
        out.update(route_E0=np.float64(res["E0"] if res["E0"] is not None else np.nan),
                   route_energies=res["energies"], route_spectral=res["spectral"],
                   route_source_norm=np.float64(res["source_norm"]))
    np.savez_compressed(os.path.join(HERE, "spectrum.npz"), **out)
    print("spectrum fixture written to", HERE)


def ramp_fixture(ref_root: str) -> None:
    """Equilibrium ramp: eq_route.solve_equilibrium(want='ramp') (eq_route.py:
    493-536) on an 8-site chain, H_builder = assemble.build_H_sparse with a
    uniform drive (assemble.py:277), n_tot = excitation count per state."""
    sys.path.insert(0, ref_root)
    from src.core.manybody import eq_route as rroute                    # eq_route.py
    from src.core.manybody import assemble as rasm                      # assemble.py
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from energy_level_b200 import configs
    n = 8
    calib = configs.calib_from_positions(configs.chain_positions(n))

    def hb(om, de):
        return rasm.build_H_sparse(calib, np.full(n, om), np.full(n, de), terms=["I1"])

    codes = np.arange(1 << n, dtype=np.int64)
    n_tot = np.asarray([bin(int(c)).count("1") for c in codes], float)
    Om_t = np.linspace(0.5, 2.5, 9)
    de_t = np.linspace(4.0, -6.0, 9)
    res = rroute.solve_equilibrium({"calib": calib, "H_builder": hb, "n_sites": n}, want="ramp",
                                   backend="ed", ramp={"Om_t": Om_t, "de_t": de_t, "L": n, "n_tot": n_tot})
    np.savez_compressed(os.path.join(HERE, "ramp.npz"), n=np.int64(n), Om_t=Om_t, de_t=de_t,
                        taus=res["taus"], gaps=res["gaps"], ns=res["ns"])
    print("ramp fixture written to", HERE)


def exchange_fixture(ref_root: str) -> None:
    """Exchange channels (I2 J, I3 A; channels.py:91-132):
    hamiltonian_linear_operator (matrix_free.py:51-62) on the full basis with
    complex J/A/Omega, on a fixed-excitation sector and on a blockade chain;
    scan_ground_sectors (sector_scan.py:61-132) of a dipolar XY chain; and a
    fixed-sector ground state through solve_equilibrium (eq_route.py:575-612)."""
    sys.path.insert(0, ref_root)
    from src.core.manybody import basis as rbasis                       # basis.py
    from src.core.manybody import matrix_free as rmf                    # matrix_free.py
    from src.core.manybody import sector_scan as rscan                  # sector_scan.py
    from src.core.manybody import eq_route as rroute                    # eq_route.py
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from energy_level_b200 import configs
    rng = np.random.default_rng(20261204)
    out = {}

    def pairs_of(n, jfun, afun, vscale):
        pos = configs.chain_positions(n, a=5.5, jitter=rng.uniform(-0.3, 0.3, n))
        ps = []
        for i in range(n):
            for j in range(i + 1, n):
                r = float(np.linalg.norm(pos[j] - pos[i]))
                ps.append({'i': i, 'j': j, 'V': vscale * configs.C6_70S / r ** 6,
                           'J': jfun(i, j, r), 'A': afun(i, j, r)})
        return {'atoms': [{'id': i, 'pos': [float(x) for x in p]} for i, p in enumerate(pos)],
                'pairs': ps}

    cases = {
        # full basis, every channel complex
        "full7": (7, None, ['I1', 'I2', 'I3'],
                  lambda i, j, r: (0.6 - 0.25j) * (5.5 / r) ** 3,
                  lambda i, j, r: (0.05 + 0.03j) if j == i + 1 else 0.0,
                  rng.uniform(0.5, 2.0, 7) * np.exp(1j * rng.uniform(0, 1, 7)), 1e-2),
        # fixed-excitation sector, real J
        "charge10_4": (10, ('charge', 4), ['I1', 'I2'],
                       lambda i, j, r: -0.7 * (5.5 / r) ** 3, lambda i, j, r: 0.0,
                       np.zeros(10), 1e-3),
        # fixed-excitation sector, complex J
        "charge9_3c": (9, ('charge', 3), ['I1', 'I2'],
                       lambda i, j, r: (0.4 + 0.3j) * (5.5 / r) ** 3, lambda i, j, r: 0.0,
                       np.zeros(9), 1e-3),
        # blockade chain: J/A targets outside the sector are dropped
        "chain10": (10, ('blockade', configs.chain_edges(10)), ['I1', 'I2', 'I3'],
                    lambda i, j, r: 0.5 * (5.5 / r) ** 3,
                    lambda i, j, r: 0.2 if j == i + 2 else 0.0,
                    rng.uniform(0.5, 2.0, 10), 1.0),
    }
    for name, (n, basis, use, jf, af, om, vs) in cases.items():
        calib = pairs_of(n, jf, af, vs)
        de = rng.uniform(-2.0, 2.0, n)
        if basis is None:
            idx = None
        elif basis[0] == 'charge':
            idx = np.asarray(rmf.number_sector_basis(n, basis[1]), np.int64)
        else:
            idx = np.asarray(rbasis.independent_states(n, basis[1]), np.int64)
        op = rmf.hamiltonian_linear_operator(calib, Om=om, delta=de, terms=use, basis_indices=idx)
        dim = op.shape[0]
        x = rng.normal(size=dim) + 1j * rng.normal(size=dim)
        out["x_" + name] = x
        out["y_" + name] = op @ x
        out["n_" + name] = np.int64(n)
        out["om_" + name] = np.asarray(om, complex)
        out["de_" + name] = de
        out["codes_" + name] = np.arange(1 << n, dtype=np.int64) if idx is None else idx
        out["pairs_" + name] = np.asarray([[p['i'], p['j']] for p in calib['pairs']], np.int64)
        out["V_" + name] = np.asarray([p['V'] for p in calib['pairs']], float)
        out["J_" + name] = np.asarray([complex(p['J']) for p in calib['pairs']], complex)
        out["A_" + name] = np.asarray([complex(p['A']) for p in calib['pairs']], complex)
        out["terms_" + name] = np.asarray(use)

    # sector scan of a dipolar XY chain (N = 10, Omega = 0)
    xy = configs.xy_chain(10)
    r = rscan.scan_ground_sectors(xy['calib'], delta=xy['delta'], Om=np.zeros(10),
                                  terms=['I1', 'I2'], device='cpu', dense_max=64)
    out["scan_E0"] = np.float64(r['E0'])
    out["scan_sector"] = np.int64(r['sector'])
    out["scan_sector_E0"] = np.asarray([row['E0'] for row in r['per_sector']], float)
    out["scan_sector_gap"] = np.asarray([row['gap'] for row in r['per_sector']], float)
    out["scan_sector_dim"] = np.asarray([row['dim'] for row in r['per_sector']], np.int64)
    out["scan_dimension_sum"] = np.int64(r['dimension_sum'])

    # fixed-sector ground state through the equilibrium route (ED backend)
    g = rroute.solve_equilibrium({'calib': xy['calib'], 'Om': np.zeros(10), 'delta': xy['delta'],
                                  'terms': ['I1', 'I2']}, want='gs', backend='ed', sector=5)
    out["gs5_E0"] = np.float64(g['E0'])
    out["gs5_gap"] = np.float64(g['gap'])
    out["gs5_n_atom"] = np.asarray(g['n_atom'], float)
    out["gs5_corr"] = np.asarray(g['corr'], float)
    out["gs5_sector_idx"] = np.asarray(g['sector_idx'], np.int64)
    np.savez_compressed(os.path.join(HERE, "exchange.npz"), **out)
    print("exchange fixture written to", HERE)


def observables_fixture(ref_root: str) -> None:
    """Spin observables and entropies: observables.spin_observables /
    spin_observables_basis (observables.py:117-205), entropy_at_cut /
    entropy_in_basis (observables.py:50-114), corr_matrix (:40-47), and two
    evolutions with every observable on (engine_ed.py:153-372): a full-basis
    XY + drive quench with segments and a projected blockade ramp."""
    sys.path.insert(0, ref_root)
    from src.core.manybody import observables as robs                   # observables.py
    from src.core.manybody import engine_ed as red                      # engine_ed.py
    from src.core.manybody import basis as rbasis                       # basis.py
    from src.core.manybody import hamiltonian_plan as rplan             # hamiltonian_plan.py
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from energy_level_b200 import configs
    rng = np.random.default_rng(20261205)
    out = {}
    # single states
    n = 7
    psi = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    psi /= np.linalg.norm(psi)
    ob = robs.spin_observables(psi, n)
    out["full_psi"] = psi
    for k in ("sx", "sy", "sz", "sp", "sm", "xy_corr", "phase"):
        out["full_" + k] = np.asarray(ob[k])
    out["full_S3"] = np.float64(robs.entropy_at_cut(psi, n, 3))
    nb = 10
    states = np.asarray(rbasis.independent_states(nb, configs.chain_edges(nb)), np.int64)
    q = rng.normal(size=states.size) + 1j * rng.normal(size=states.size)
    q /= np.linalg.norm(q)
    ob = robs.spin_observables_basis(q, states, nb)
    out["basis_psi"] = q
    out["basis_states"] = states
    for k in ("sx", "sy", "sz", "sp", "sm", "xy_corr", "phase"):
        out["basis_" + k] = np.asarray(ob[k])
    out["basis_S5"] = np.float64(robs.entropy_in_basis(q, states, nb, 5))
    bits = np.asarray([((states >> (nb - 1 - i)) & 1) for i in range(nb)], float)
    out["basis_corr"] = robs.corr_matrix(bits, np.abs(q) ** 2)

    # evolution 1: full basis, XY exchange + drive, three segments
    n = 6
    xy = configs.xy_chain(n, seed=21)
    segs = [{"t0": 0.0, "Om": np.full(n, 0.8), "delta": xy["delta"]},
            {"t0": 150.0, "Om": np.full(n, 1.2), "delta": xy["delta"] - 0.5},
            {"t0": 300.0, "Om": np.full(n, 0.4), "delta": xy["delta"] + 0.3}]
    t = np.linspace(0.0, 400.0, 6)
    r = red.evolve_manybody(xy["calib"], psi0="rg" * (n // 2), t_grid=t, segments=segs, terms=["I1", "I2"],
                            record_psi=True, link_pairs=[(0, 1), (2, 4)])
    out["ev1_n"] = np.int64(n)
    out["ev1_t"] = t
    out["ev1_seg_t0"] = np.asarray([sg["t0"] for sg in segs])
    out["ev1_seg_om"] = np.asarray([sg["Om"] for sg in segs])
    out["ev1_seg_de"] = np.asarray([sg["delta"] for sg in segs])
    for k in ("pops_atom", "S", "corr", "norms", "pops", "basis_probabilities", "psi_amp"):
        out["ev1_" + k] = np.asarray(r[k])
    for k in ("sx", "sy", "sz", "sp", "sm", "phase", "xy_corr", "link_corr"):
        out["ev1_obs_" + k] = np.asarray(r["observables"][k])

    # evolution 2: projected blockade chain, two segments
    n = 10
    calib = configs.calib_from_positions(configs.chain_positions(n))
    segs = [{"t0": 0.0, "Om": np.full(n, 2.0), "delta": np.full(n, 3.0)},
            {"t0": 100.0, "Om": np.full(n, 1.5), "delta": np.full(n, -2.0)}]
    plan = rplan.build_plan(calib, Om=np.full(n, 2.0), delta=np.zeros(n), terms=["I1"],
                            constraint={"kind": "blockade", "edges": configs.chain_edges(n)})
    t = np.linspace(0.0, 200.0, 5)
    r = red.evolve_manybody(calib, psi0="g" * n, t_grid=t, segments=segs, plan=plan, terms=["I1"],
                            record_psi=True)
    out["ev2_n"] = np.int64(n)
    out["ev2_t"] = t
    out["ev2_seg_t0"] = np.asarray([sg["t0"] for sg in segs])
    out["ev2_seg_om"] = np.asarray([sg["Om"] for sg in segs])
    out["ev2_seg_de"] = np.asarray([sg["delta"] for sg in segs])
    out["ev2_states"] = np.asarray(r["basis_states"], np.int64)
    for k in ("pops_atom", "S", "corr", "norms", "pops", "basis_probabilities", "psi_amp"):
        out["ev2_" + k] = np.asarray(r[k])
    for k in ("sx", "sy", "sz", "sp", "sm", "phase", "xy_corr"):
        out["ev2_obs_" + k] = np.asarray(r["observables"][k])
    np.savez_compressed(os.path.join(HERE, "observables.npz"), **out)
    print("observables fixture written to", HERE)


def loss_fixture(ref_root: str) -> None:
    """Loss rates gamma (non-Hermitian diagonal, channels.py:69-76):
    hamiltonian_linear_operator with gamma on a full basis and on a blockade
    chain, and evolve_manybody (engine_ed.py:153-372) with gamma: full basis
    with XY exchange and three segments, projected chain with a static drive
    (the expm_multiply path of engine_ed.py:117-127)."""
    sys.path.insert(0, ref_root)
    from src.core.manybody import matrix_free as rmf                    # matrix_free.py
    from src.core.manybody import engine_ed as red                      # engine_ed.py
    from src.core.manybody import basis as rbasis                       # basis.py
    from src.core.manybody import hamiltonian_plan as rplan             # hamiltonian_plan.py
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from energy_level_b200 import configs
    rng = np.random.default_rng(20261206)
    out = {}
    for name, n, edges in (("full7", 7, None), ("chain10", 10, configs.chain_edges(10))):
        calib = configs.calib_from_positions(configs.chain_positions(n))
        om = rng.uniform(0.5, 2.0, n)
        de = rng.uniform(-2.0, 2.0, n)
        ga = rng.uniform(0.0, 5.0, n)
        idx = None if edges is None else np.asarray(rbasis.independent_states(n, edges), np.int64)
        op = rmf.hamiltonian_linear_operator(calib, Om=om, delta=de, gamma=ga, terms=["I1"], basis_indices=idx)
        x = rng.normal(size=op.shape[0]) + 1j * rng.normal(size=op.shape[0])
        out["hv_" + name + "_x"] = x
        out["hv_" + name + "_y"] = op @ x
        out["hv_" + name + "_om"] = om
        out["hv_" + name + "_de"] = de
        out["hv_" + name + "_ga"] = ga
    # evolution 1: full basis, XY + drive, three segments, loss
    n = 6
    xy = configs.xy_chain(n, seed=31)
    ga = np.linspace(2.0, 8.0, n)
    segs = [{"t0": 0.0, "Om": np.full(n, 0.9), "delta": xy["delta"]},
            {"t0": 120.0, "Om": np.full(n, 1.4), "delta": xy["delta"] - 0.4},
            {"t0": 260.0, "Om": np.full(n, 0.5), "delta": xy["delta"] + 0.2}]
    t = np.linspace(0.0, 400.0, 6)
    r = red.evolve_manybody(xy["calib"], psi0="rg" * (n // 2), t_grid=t, segments=segs, gamma=ga,
                            terms=["I1", "I2"], record_psi=True)
    out["ev1_t"] = t
    out["ev1_ga"] = ga
    out["ev1_seg_t0"] = np.asarray([sg["t0"] for sg in segs])
    out["ev1_seg_om"] = np.asarray([sg["Om"] for sg in segs])
    out["ev1_seg_de"] = np.asarray([sg["delta"] for sg in segs])
    for k in ("pops_atom", "norms", "loss", "S", "corr", "psi_amp"):
        out["ev1_" + k] = np.asarray(r[k])
    out["ev1_backend"] = np.asarray(r["backend"])
    # evolution 2: projected blockade chain, static drive, loss
    n = 9
    calib = configs.calib_from_positions(configs.chain_positions(n))
    plan = rplan.build_plan(calib, Om=np.full(n, 2.0), delta=np.full(n, -1.0), terms=["I1"],
                            constraint={"kind": "blockade", "edges": configs.chain_edges(n)})
    ga = np.full(n, 3.0)
    t = np.linspace(0.0, 300.0, 4)
    r = red.evolve_manybody(calib, psi0="g" * n, t_grid=t, Om=np.full(n, 2.0), delta=np.full(n, -1.0),
                            gamma=ga, plan=plan, terms=["I1"], record_psi=True)
    out["ev2_t"] = t
    out["ev2_ga"] = ga
    out["ev2_states"] = np.asarray(r["basis_states"], np.int64)
    for k in ("pops_atom", "norms", "loss", "S", "corr", "psi_amp"):
        out["ev2_" + k] = np.asarray(r[k])
    np.savez_compressed(os.path.join(HERE, "loss.npz"), **out)
    print("loss fixture written to", HERE)


def constraint_fixture(ref_root: str) -> None:
    """Plans from constraint specs (hamiltonian_plan.py:15-50 _constraint_dict
    / _edges, build_plan :53-72) on a 3x4 square lattice (a = 6 um, C6/r^6
    pairs): blockade and pxp in project mode with edges from |V| >=
    threshold_mhz (nearest and diagonal neighbours at 2 MHz: a general graph,
    not a chain or ring; nearest neighbours only at 10 MHz), 'auto' edges and
    mode='full'; each with the reference's ground state on its plan
    (equilibrium.ground_state on compile_sparse, dense eigh), and the
    refusal of a projecting spec with neither edges nor a threshold."""
    import json
    sys.path.insert(0, ref_root)
    from src.core.manybody import equilibrium as req
    from src.core.manybody import hamiltonian_plan as rplan
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from energy_level_b200 import configs
    pos = [[6.0 * m, 6.0 * k, 0.0] for m in range(3) for k in range(4)]
    n = len(pos)
    calib = configs.calib_from_positions(pos)
    rng = np.random.default_rng(11)
    om = rng.uniform(1.0, 2.5, n)
    de = rng.uniform(-2.0, 2.0, n)
    specs = {"blockade_thr": {"kind": "blockade", "threshold_mhz": 2.0},
             "pxp_auto": {"kind": "pxp", "edges": "auto", "threshold_mhz": 2.0},
             "blockade_nn": {"kind": "blockade", "threshold_mhz": 10.0},
             "blockade_full": {"kind": "blockade", "mode": "full", "threshold_mhz": 2.0}}
    out = dict(pos=np.asarray(pos), om=om, de=de, names=np.asarray(list(specs)))
    for name, spec in specs.items():
        plan = rplan.build_plan(calib, Om=om, delta=de, terms=["I1"], constraint=spec)
        gs = req.ground_state(rplan.compile_sparse(plan), dense_max=1 << 13, k=2)
        out[name + "_spec"] = np.asarray(json.dumps(spec))
        out[name + "_projected"] = np.asarray(bool(plan["projected"]))
        out[name + "_edges"] = np.asarray(plan["blockade_edges"], np.int64).reshape(-1, 2)
        out[name + "_dim"] = np.int64(plan["dim"])
        out[name + "_states"] = np.asarray(plan["states"] if plan["states"] is not None else [], np.int64)
        out[name + "_E0"] = np.float64(gs["E0"])
        out[name + "_gap"] = np.float64(gs["gap"])
    try:
        rplan.build_plan(calib, Om=om, delta=de, terms=["I1"], constraint={"kind": "blockade"})
        out["refusal"] = np.asarray("")
    except ValueError as e:
        out["refusal"] = np.asarray(str(e))
    np.savez_compressed(os.path.join(HERE, "constraint.npz"), **out)
    print("constraint fixture written to", HERE)


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: make_golden.py <reference checkout> [all|spectrum|ramp|exchange|observables|loss|constraint]")
    root = sys.argv[1]
    which = sys.argv[2] if len(sys.argv) > 2 else "all"
    if which == "spectrum":
        spectrum_fixture(root)
    elif which == "ramp":
        ramp_fixture(root)
    elif which == "exchange":
        exchange_fixture(root)
    elif which == "observables":
        observables_fixture(root)
    elif which == "loss":
        loss_fixture(root)
    elif which == "constraint":
        constraint_fixture(root)
    else:
        main(root)
        spectrum_fixture(root)
        ramp_fixture(root)
        exchange_fixture(root)
        observables_fixture(root)
        loss_fixture(root)
        constraint_fixture(root)
